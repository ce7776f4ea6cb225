// sv_batch.cu — batched engine: thousands of independent circuits of uneven width
// in one persistent launch.
//
// Each CTA pulls circuits from an atomic work queue (longest first).  A circuit
// whose state fits in shared memory (2^n <= 2^kt amplitudes per live state) runs
// entirely on chip: |0...0> is created in shared memory, every gate is applied
// there and only the expectation values (or gradients) leave the SM.  Wider
// circuits run as a host-planned list of segments: each segment is a run of
// gates whose wires fit in kt local bits, executed as one HBM/L2 pass over the
// 2^(n-kt) tiles of the state, every tile staged in shared memory.
//
// Differentiation is the adjoint method of LQ/algorithms/AdjointJacobianLQubit.hpp:212-335
// restricted to the vector-Jacobian product (one bra = sum_o dy_o O_o psi, the
// trick of lightning_qubit.py:747-772): per circuit two live states (lambda and
// the bra), a reverse sweep applying U^dagger to both and, for each differentiated
// gate, the FP64 product -2 * scale * Im<bra|G|lambda> accumulated per warp and
// reduced in a fixed order by a second kernel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/b200sv.h"
#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace batch {

// F_PAIR4: the double-excitation family, a 2x2 block on rows 0011 / 1100 of each 16-row group of
// four target bits, the other rows scaled by gamma.  F_MATK: a constant dense matrix on 3 or 4
// target bits.  For both, off[j] holds the single bit of target j (matrix order, j = 0 the most
// significant) instead of row offsets.
enum Form : uint8_t { F_MAT1 = 1, F_MAT2 = 2, F_DIAG = 3, F_SWAP = 4, F_PARITY = 5, F_NOOP = 6, F_PAIR4 = 7, F_MATK = 8 };
// G_PAIR4: generator of a double excitation, Y on rows 0011 / 1100 and gk (0: 0, 1: +1, 2: -1)
// times the identity on the other rows
enum GForm : uint8_t { G_NONE = 0, G_MAT = 1, G_PARITY = 2, G_PAIR4 = 3 };
constexpr uint8_t kConstGate = 255;
constexpr int kMaxKt = 14;
constexpr int kObsPerPass = 16;  // observables whose expectation values one forward pass accumulates

// One gate with bit positions local to its segment's tile.
struct DOp {
    uint8_t form, gate, nb, inv;
    uint8_t nt, gform, gnb, gk;
    uint8_t maxbit;      // highest tile bit the gate (or its generator) touches
    uint8_t run;         // >= 2: first of `run` single-wire gates on bit `rbit` fused into one pass
    uint8_t rbit;
    uint8_t gcode;       // run members' generator: 1 X, 2 Y, 3 Z, 4 |1><1| (0: none / general)
    uint8_t mkind;       // run members' matrix structure (MK_* below)
    uint8_t pair;        // forward run heads: pairing code with the next run (pair_sig)
    uint16_t low[4];     // insertion masks of the gate bits (ascending)
    uint16_t glow[2];    // insertion masks of the generator bits
    uint32_t cmask;      // control bits (must be set)
    uint32_t off[4];     // row offsets of the targets (row r: bit (nt-1-j) <-> target j)
    uint32_t goff[4];    // generator row offsets
    uint32_t pmask;      // parity bits (MultiRZ)
    int32_t pslot;       // parameter slot, -1 for constant gates
    int32_t gslot;       // gradient slot, -1 when not differentiated
    uint32_t cidx;       // constant coefficients (consts[cidx*16..])
    uint32_t gcidx;      // generator matrix (consts[gcidx*16..])
    uint8_t back;        // run members: distance back to the run's head (0 for heads and single gates)
    double gscale;       // -2 * generator scale * (inverse ? -1 : 1)
};
static_assert(sizeof(DOp) == 96, "DOp layout: op records are staged in shared memory");

struct DSeg {
    uint32_t op_begin, nops;
    uint8_t lbits[kMaxKt];   // tile bit j -> state bit (ascending)
    uint8_t gbits[40];       // tile index bit j -> state bit (ascending)
    uint8_t nl, ng;
};

static_assert(sizeof(DSeg) % 4 == 0, "segments are staged in shared memory as 32-bit words");

struct DCirc {
    uint32_t n, kt, resident;
    uint32_t seg_begin, nseg;
    uint64_t off_a, off_b;   // offsets into the state pools (amplitudes)
    uint32_t term_begin, nterms;
    uint32_t nobs, out_begin;
};

struct DTerm {
    uint32_t obs;
    int32_t ny;
    double coeff;
    uint64_t xmask, zmask;
};

constexpr int kMaxRun = 3;
constexpr int kMaxSegOpsStaged = 160;  // ops of a segment staged in shared memory (planner cap)
// structure of a single-wire matrix, used to spend fewer instructions per amplitude pair
enum MKind : uint8_t { MK_GENERAL = 0, MK_DIAG = 1, MK_PHASE1 = 2, MK_REAL = 3, MK_SWAP = 4, MK_RX = 5 };

// single complex product m * v (FMA-formed components)
template <typename R> __device__ __forceinline__ C<R> cmul1(C<R> m, C<R> v) {
    return mk<R>(fma(m.x, v.x, -(m.y * v.y)), fma(m.x, v.y, m.y * v.x));
}
// a*x + b*y for real coefficients, accurate to about one rounding: the product b*y is
// split exactly with an FMA (TwoProduct) and its error added back after the second FMA.
template <typename R> __device__ __forceinline__ R dot2r(R a, R x, R b, R y) {
    const R w = b * y;
    const R e = fma(b, y, -w);
    return fma(a, x, w) + e;
}

// Apply a single-wire matrix m with structure KIND to the pair (v0, v1) in place.
template <typename R, int KIND>
__device__ __forceinline__ void apply_pair_k(const C<R> (&m)[4], C<R> &v0, C<R> &v1) {
    if constexpr (KIND == MK_DIAG) {
        v0 = cmul1<R>(m[0], v0);
        v1 = cmul1<R>(m[3], v1);
    } else if constexpr (KIND == MK_PHASE1) {
        v1 = cmul1<R>(m[3], v1);
    } else if constexpr (KIND == MK_SWAP) {
        const C<R> t = v0;
        v0 = v1;
        v1 = t;
    } else if constexpr (KIND == MK_REAL) {  // m real
        const C<R> a = v0, b = v1;
        v0 = mk<R>(dot2r<R>(m[0].x, a.x, m[1].x, b.x), dot2r<R>(m[0].x, a.y, m[1].x, b.y));
        v1 = mk<R>(dot2r<R>(m[2].x, a.x, m[3].x, b.x), dot2r<R>(m[2].x, a.y, m[3].x, b.y));
    } else if constexpr (KIND == MK_RX) {  // real diagonal, imaginary off-diagonal
        const C<R> a = v0, b = v1;
        v0 = mk<R>(dot2r<R>(m[0].x, a.x, -m[1].y, b.y), dot2r<R>(m[0].x, a.y, m[1].y, b.x));
        v1 = mk<R>(dot2r<R>(-m[2].y, a.y, m[3].x, b.x), dot2r<R>(m[2].y, a.x, m[3].x, b.y));
    } else {
        CAcc<R> p, q;
        p.set(m[0], v0); p.add(m[1], v1);
        q.set(m[2], v0); q.add(m[3], v1);
        v0 = p.get();
        v1 = q.get();
    }
}

// the same with the structure known only at run time (uniform across the block)
template <typename R> __device__ __forceinline__ void apply_pair(int kind, const C<R> (&m)[4], C<R> &v0, C<R> &v1) {
    switch (kind) {
    case MK_DIAG: apply_pair_k<R, MK_DIAG>(m, v0, v1); break;
    case MK_PHASE1: apply_pair_k<R, MK_PHASE1>(m, v0, v1); break;
    case MK_SWAP: apply_pair_k<R, MK_SWAP>(m, v0, v1); break;
    case MK_REAL: apply_pair_k<R, MK_REAL>(m, v0, v1); break;
    case MK_RX: apply_pair_k<R, MK_RX>(m, v0, v1); break;
    default: apply_pair_k<R, MK_GENERAL>(m, v0, v1); break;
    }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ins_local(uint32_t g, const uint16_t *low, int nb) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (j < nb) {
            const uint32_t lo = g & low[j];
            g = ((g ^ lo) << 1) | lo;
        }
    }
    return g;
}

// Per-parameter trigonometry, computed once per launch: (cos t/2, sin t/2, cos t, sin t).
__global__ void k_trig(const double *__restrict__ params, uint64_t n, double4 *__restrict__ cs) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        double s, c, s2, c2;
        sincos(0.5 * params[p], &s, &c);
        sincos(params[p], &s2, &c2);
        cs[p] = make_double4(c, s, c2, s2);
    }
}

// Coefficients of a gate (or of its adjoint): MAT1 -> 4, MAT2 -> 16, DIAG -> 2^nt, PARITY -> 2.
// NM: 16 for two-wire dense steps (F_MAT2), 4 for every other form; an array of exactly
// that size keeps the coefficients of the common steps in few registers.
template <typename R, int NM>
__device__ __forceinline__ void op_coeffs(const DOp &op, const double4 *__restrict__ cs,
                                          const double2 *__restrict__ consts, bool adj, C<R> (&m)[NM]) {
    if (op.gate == kConstGate) {
        const double2 *c = consts + (size_t)op.cidx * 16;
        // NM == 4: D is 2 at compile time; NM == 16 serves every form (D chosen at run time)
        const int D = (NM == 16 && op.form == F_MAT2) ? 4 : 2;
        if (op.form == F_MAT1 || (NM == 16 && (op.form == F_MAT2 || op.form == F_PAIR4))) {
            for (int r = 0; r < D; ++r)
                for (int q = 0; q < D; ++q) {
                    const double2 z = adj ? c[q * D + r] : c[r * D + q];
                    m[r * D + q] = mk<R>((R)z.x, (R)(adj ? -z.y : z.y));
                }
            if constexpr (NM == 16) {
                if (op.form == F_PAIR4) m[4] = mk<R>((R)c[4].x, (R)(adj ? -c[4].y : c[4].y));  // gamma
            }
        } else {
            for (int r = 0; r < 4; ++r) m[r] = mk<R>((R)c[r].x, (R)(adj ? -c[r].y : c[r].y));
        }
        return;
    }
    const double4 q = cs[op.pslot];
    const double sg = ((op.inv != 0) != adj) ? -1.0 : 1.0;
    const R cr = (R)q.x, sr = (R)(sg * q.y), z = (R)0, one = (R)1;
    switch (op.gate) {
    case B200SV_RX: case B200SV_CRX:
        m[0] = mk<R>(cr, z); m[1] = mk<R>(z, -sr); m[2] = mk<R>(z, -sr); m[3] = mk<R>(cr, z); break;
    case B200SV_RY: case B200SV_CRY:
        m[0] = mk<R>(cr, z); m[1] = mk<R>(-sr, z); m[2] = mk<R>(sr, z); m[3] = mk<R>(cr, z); break;
    case B200SV_RZ: case B200SV_CRZ: case B200SV_MultiRZ:
        m[0] = mk<R>(cr, -sr); m[1] = mk<R>(cr, sr); break;
    case B200SV_PhaseShift: case B200SV_ControlledPhaseShift:
        m[0] = mk<R>((R)q.z, (R)(sg * q.w)); break;
    case B200SV_IsingZZ:
        m[0] = mk<R>(cr, -sr); m[1] = mk<R>(cr, sr); m[2] = mk<R>(cr, sr); m[3] = mk<R>(cr, -sr); break;
    case B200SV_DoubleExcitation: case B200SV_DoubleExcitationMinus: case B200SV_DoubleExcitationPlus:
        if constexpr (NM == 16) {  // block on rows (0011, 1100), gamma on the others
            m[0] = mk<R>(cr, z); m[1] = mk<R>(-sr, z); m[2] = mk<R>(sr, z); m[3] = mk<R>(cr, z);
            m[4] = op.gate == B200SV_DoubleExcitationMinus  ? mk<R>(cr, -sr)
                   : op.gate == B200SV_DoubleExcitationPlus ? mk<R>(cr, sr)
                                                            : mk<R>(one, z);
        }
        break;
    default: {
        if constexpr (NM == 16) {  // two-wire dense gates (F_MAT2)
#pragma unroll
            for (int i = 0; i < NM; ++i) m[i] = mk<R>(z, z);
            if (op.gate == B200SV_IsingXX) {
                m[0] = m[5] = m[10] = m[15] = mk<R>(cr, z);
                m[3] = m[6] = m[9] = m[12] = mk<R>(z, -sr);
            } else if (op.gate == B200SV_IsingYY) {
                m[0] = m[5] = m[10] = m[15] = mk<R>(cr, z);
                m[3] = m[12] = mk<R>(z, sr);
                m[6] = m[9] = mk<R>(z, -sr);
            } else if (op.gate == B200SV_IsingXY) {
                m[0] = m[15] = mk<R>(one, z);
                m[5] = m[10] = mk<R>(cr, z);
                m[6] = m[9] = mk<R>(z, sr);
            } else {  // SingleExcitation (+/-)
                m[5] = m[10] = mk<R>(cr, z);
                m[6] = mk<R>(-sr, z);
                m[9] = mk<R>(sr, z);
                C<R> e = mk<R>(one, z);
                if (op.gate == B200SV_SingleExcitationMinus) e = mk<R>(cr, -sr);
                if (op.gate == B200SV_SingleExcitationPlus) e = mk<R>(cr, sr);
                m[0] = m[15] = e;
            }
        }
    }
    }
}

// 2x2 matrix of a run member (single-wire gate on the run bit), or of its adjoint.
template <typename R>
__device__ __forceinline__ void member_mat(const DOp &op, const double4 *__restrict__ cs,
                                           const double2 *__restrict__ consts, bool adj, C<R> (&m)[4]) {
    const C<R> zero = mk<R>(0, 0), one = mk<R>(1, 0);
    if (op.form == F_SWAP) {
        m[0] = zero; m[1] = one; m[2] = one; m[3] = zero;
        return;
    }
    C<R> t[4];
    op_coeffs<R, 4>(op, cs, consts, adj, t);
    if (op.form == F_MAT1) {
        m[0] = t[0]; m[1] = t[1]; m[2] = t[2]; m[3] = t[3];
    } else if (op.nt == 1) {  // diagonal on the bit
        m[0] = t[0]; m[1] = zero; m[2] = zero; m[3] = t[1];
    } else {                  // phase on |1> of the bit
        m[0] = one; m[1] = zero; m[2] = zero; m[3] = t[0];
    }
}

// The same from the op's precomputed coefficients t (op_coeffs<R, 4> in the same direction).
template <typename R>
__device__ __forceinline__ void member_from(const DOp &op, const C<R> (&t)[4], C<R> (&m)[4]) {
    const C<R> zero = mk<R>(0, 0), one = mk<R>(1, 0);
    if (op.form == F_SWAP) {
        m[0] = zero; m[1] = one; m[2] = one; m[3] = zero;
    } else if (op.form == F_MAT1) {
        m[0] = t[0]; m[1] = t[1]; m[2] = t[2]; m[3] = t[3];
    } else if (op.nt == 1) {
        m[0] = t[0]; m[1] = zero; m[2] = zero; m[3] = t[1];
    } else {
        m[0] = one; m[1] = zero; m[2] = zero; m[3] = t[0];
    }
}

// Iteration range of a step's groups: warp-local steps (every touched bit below
// wl) keep each warp inside its own 2^wl-amplitude block, so consecutive
// warp-local steps only need __syncwarp; other steps spread over the block.
struct Range {
    uint32_t g0, g1, gs;
};
__device__ __forceinline__ Range groups(int kt, int wl, int nb, bool wloc) {
    Range r;
    if (wloc) {
        const uint32_t per = 1u << (wl - nb);
        r.g0 = (threadIdx.x >> 5) * per + (threadIdx.x & 31);
        r.g1 = ((threadIdx.x >> 5) + 1) * per;
        r.gs = 32;
    } else {
        r.g0 = threadIdx.x;
        r.g1 = 1u << (kt - nb);
        r.gs = blockDim.x;
    }
    return r;
}

// two-wire dense step (F_MAT2) with its 16 coefficients
template <typename R, int NS>
__device__ __forceinline__ void apply_mat2(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                           const C<R> (&m)[16]) {
    const Range rg = groups(kt, wl, op.nb, wloc);
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t base = ins_local(g, op.low, op.nb) | op.cmask;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            C<R> *t = s[q];
            C<R> v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) v[r] = t[base + op.off[r]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                CAcc<R> a;
#pragma unroll
                for (int c = 0; c < 4; ++c) cacc_term<R>(a, c, m[r * 4 + c], v[c]);
                t[base + op.off[r]] = a.get();
            }
        }
    }
}

// apply one gate of any other form (coefficients already adjointed when needed) to NS tiles
template <typename R, int NS>
__device__ __forceinline__ void apply_op(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                         const C<R> (&m)[4]) {
    if (op.form == F_NOOP) return;
    if (op.form == F_PARITY) {
        const Range rg = groups(kt, wl, 0, wloc);
        for (uint32_t i = rg.g0; i < rg.g1; i += rg.gs) {
            const C<R> f = (__popc(i & op.pmask) & 1) ? m[1] : m[0];
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                CAcc<R> a;
                a.set(f, s[q][i]);
                s[q][i] = a.get();
            }
        }
        return;
    }
    const Range rg = groups(kt, wl, op.nb, wloc);
    if (op.form == F_SWAP && op.nb == 2) {  // CNOT, SWAP: two inserted bits, masks held in registers
        const uint32_t l0 = op.low[0], l1 = op.low[1], cm = op.cmask, oa = op.off[0], ob = op.off[1];
        for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
            uint32_t lo = g & l0;
            uint32_t i = ((g ^ lo) << 1) | lo;
            lo = i & l1;
            i = (((i ^ lo) << 1) | lo) | cm;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                C<R> *t = s[q];
                const C<R> a = t[i + oa];
                t[i + oa] = t[i + ob];
                t[i + ob] = a;
            }
        }
        return;
    }
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t base = ins_local(g, op.low, op.nb) | op.cmask;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            C<R> *t = s[q];
            switch (op.form) {
            case F_MAT1: {
                const C<R> v0 = t[base + op.off[0]], v1 = t[base + op.off[1]];
                CAcc<R> a, b;
                a.set(m[0], v0); a.add(m[1], v1);
                b.set(m[2], v0); b.add(m[3], v1);
                t[base + op.off[0]] = a.get();
                t[base + op.off[1]] = b.get();
                break;
            }
            case F_DIAG: {
                const int rows = 1 << op.nt;
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    if (r < rows) {
                        CAcc<R> a;
                        a.set(m[r], t[base + op.off[r]]);
                        t[base + op.off[r]] = a.get();
                    }
                }
                break;
            }
            case F_SWAP: {
                const C<R> a = t[base + op.off[0]];
                t[base + op.off[0]] = t[base + op.off[1]];
                t[base + op.off[1]] = a;
                break;
            }
            default: break;
            }
        }
    }
}

// offset of row r of a group of K target bits whose single bits are off[0..K-1] (off[0] the most
// significant matrix-index bit)
template <int K>
__device__ __forceinline__ uint32_t row_offset(const uint32_t *off, int r) {
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < K; ++j)
        if ((r >> (K - 1 - j)) & 1) o |= off[j];
    return o;
}

// double-excitation step (F_PAIR4): m[0..3] on rows 0011 / 1100 of each 16-row group, the
// other 14 rows times gamma = m[4] (skipped when gamma is exactly 1)
template <typename R, int NS>
__device__ __forceinline__ void apply_pair4(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                            const C<R> (&m)[16]) {
    const Range rg = groups(kt, wl, 4, wloc);
    const uint32_t opa = op.off[2] | op.off[3], opb = op.off[0] | op.off[1];
    const bool phase = !(m[4].x == (R)1 && m[4].y == (R)0);
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t base = ins_local(g, op.low, 4) | op.cmask;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            C<R> *t = s[q];
            const C<R> a = t[base + opa], b = t[base + opb];
            CAcc<R> x, y;
            x.set(m[0], a); x.add(m[1], b);
            y.set(m[2], a); y.add(m[3], b);
            t[base + opa] = x.get();
            t[base + opb] = y.get();
            if (phase) {
#pragma unroll
                for (int r = 0; r < 16; ++r) {
                    if (r == 3 || r == 12) continue;
                    const uint32_t o = base + row_offset<4>(op.off, r);
                    CAcc<R> w;
                    w.set(m[4], t[o]);
                    t[o] = w.get();
                }
            }
        }
    }
}

// constant dense matrix on K = 3 or 4 target bits (F_MATK), coefficients read from the constant
// pool (row-major, 4^K entries), conjugate-transposed for the adjoint
template <typename R, int NS, int K>
__device__ __forceinline__ void apply_matk_k(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                             const double2 *__restrict__ consts, bool adj) {
    constexpr int D = 1 << K;
    const double2 *cm = consts + (size_t)op.cidx * 16;
    const Range rg = groups(kt, wl, op.nb, wloc);
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t base = ins_local(g, op.low, op.nb) | op.cmask;
#pragma unroll 1
        for (int q = 0; q < NS; ++q) {
            C<R> *t = s[q];
            C<R> v[D];
#pragma unroll
            for (int c = 0; c < D; ++c) v[c] = t[base + row_offset<K>(op.off, c)];
#pragma unroll 1
            for (int r = 0; r < D; ++r) {
                CAcc<R> a;
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    const double2 z = adj ? cm[c * D + r] : cm[r * D + c];
                    cacc_term<R>(a, c, mk<R>((R)z.x, (R)(adj ? -z.y : z.y)), v[c]);
                }
                t[base + row_offset<K>(op.off, r)] = a.get();
            }
        }
    }
}
template <typename R, int NS>
__device__ __forceinline__ void apply_matk(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                           const double2 *__restrict__ consts, bool adj) {
    if (op.nt == 3) apply_matk_k<R, NS, 3>(s, kt, wl, wloc, op, consts, adj);
    else apply_matk_k<R, NS, 4>(s, kt, wl, wloc, op, consts, adj);
}

// apply a step of any form with coefficients in a 16-entry array (kernels built with the
// two-wire dense paths); the parity phase is picked by index, as those kernels keep the
// array in local memory anyway
template <typename R, int NS>
__device__ __forceinline__ void apply_op_general(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp &op,
                                                 const C<R> (&m)[16]) {
    if (op.form == F_MAT2) {
        apply_mat2<R, NS>(s, kt, wl, wloc, op, m);
        return;
    }
    if (op.form == F_PAIR4) {
        apply_pair4<R, NS>(s, kt, wl, wloc, op, m);
        return;
    }
    if (op.form == F_PARITY) {
        const Range rg = groups(kt, wl, 0, wloc);
        for (uint32_t i = rg.g0; i < rg.g1; i += rg.gs) {
            const C<R> f = m[__popc(i & op.pmask) & 1];
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                CAcc<R> a;
                a.set(f, s[q][i]);
                s[q][i] = a.get();
            }
        }
        return;
    }
    const C<R>(&m4)[4] = reinterpret_cast<const C<R>(&)[4]>(m);
    apply_op<R, NS>(s, kt, wl, wloc, op, m4);
}

template <typename R, int CODE>
__device__ __forceinline__ double pair_gen_im_k(C<R> a0, C<R> a1, C<R> b0, C<R> b1);

// per-thread part of Im<bra|G|ket> on one tile, FP64
// sum over groups of Im(conj(bra) . G ket) for a 2^K x 2^K generator G (FP64)
template <typename R, int K>
__device__ __forceinline__ double gen_inner_k(const C<R> *bra, const C<R> *ket, const Range &rg, const DOp &op,
                                              const double2 *__restrict__ G) {
    constexpr int D = 1 << K;
    double acc = 0.0;
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t base = ins_local(g, op.glow, op.gnb);
        double2 v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = widen<R>(ket[base + op.goff[r]]);
#pragma unroll
        for (int r = 0; r < D; ++r) {
            double wr = 0, wi = 0;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const double2 x = G[r * D + c];
                wr += x.x * v[c].x - x.y * v[c].y;
                wi += x.x * v[c].y + x.y * v[c].x;
            }
            const double2 b = widen<R>(bra[base + op.goff[r]]);
            acc += b.x * wi - b.y * wr;
        }
    }
    return acc;
}

// FULL: the batch holds two-wire dense steps or generators (compiled only into the full kernel)
template <typename R, bool FULL>
__device__ __forceinline__ double gen_inner(const C<R> *bra, const C<R> *ket, int kt, int wl, bool wloc, const DOp &op,
                                            const double2 *__restrict__ consts) {
    double acc = 0.0;
    if (op.gform == G_PARITY) {
        const Range rg = groups(kt, wl, 0, wloc);
        for (uint32_t i = rg.g0; i < rg.g1; i += rg.gs) {
            const double2 k = widen<R>(ket[i]), b = widen<R>(bra[i]);
            const double sg = (__popc(i & op.pmask) & 1) ? -1.0 : 1.0;
            acc += sg * (b.x * k.y - b.y * k.x);
        }
        return acc;
    }
    if constexpr (FULL) {
        if (op.gform == G_PAIR4) {
            // Y on rows (0011, 1100); gamma_g times the identity on the other rows
            const Range rg = groups(kt, wl, 4, wloc);
            const uint32_t opa = op.off[2] | op.off[3], opb = op.off[0] | op.off[1];
            const double gg = op.gk == 1 ? 1.0 : op.gk == 2 ? -1.0 : 0.0;
            for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
                const uint32_t base = ins_local(g, op.low, 4) | op.cmask;
                acc += pair_gen_im_k<R, 2>(ket[base + opa], ket[base + opb], bra[base + opa], bra[base + opb]);
                if (gg != 0.0) {
                    double o = 0.0;
#pragma unroll
                    for (int r = 0; r < 16; ++r) {
                        if (r == 3 || r == 12) continue;
                        const uint32_t i = base + row_offset<4>(op.off, r);
                        const double2 k = widen<R>(ket[i]), b = widen<R>(bra[i]);
                        o += b.x * k.y - b.y * k.x;
                    }
                    acc += gg * o;
                }
            }
            return acc;
        }
    }
    const double2 *G = consts + (size_t)op.gcidx * 16;
    const Range rg = groups(kt, wl, op.gnb, wloc);
    if constexpr (FULL) {
        // general size (one or two wires), loops over the run-time size
        const int D = 1 << op.gk;
        for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
            const uint32_t base = ins_local(g, op.glow, op.gnb);
            double2 v[4];
            for (int r = 0; r < D; ++r) v[r] = widen<R>(ket[base + op.goff[r]]);
            for (int r = 0; r < D; ++r) {
                double wr = 0, wi = 0;
                for (int c = 0; c < D; ++c) {
                    const double2 x = G[r * D + c];
                    wr += x.x * v[c].x - x.y * v[c].y;
                    wi += x.x * v[c].y + x.y * v[c].x;
                }
                const double2 b = widen<R>(bra[base + op.goff[r]]);
                acc += b.x * wi - b.y * wr;
            }
        }
        return acc;
    }
    return gen_inner_k<R, 1>(bra, ket, rg, op, G);
}

__device__ __forceinline__ void add_grad(double *gradw, int32_t gslot, double p, bool first) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) p += __shfl_down_sync(0xffffffffu, p, off);
    if ((threadIdx.x & 31) == 0) {
        double *slot = gradw + (size_t)gslot * (blockDim.x >> 5) + (threadIdx.x >> 5);
        *slot = first ? p : *slot + p;
    }
}

// Im(conj(b) . G a) over one amplitude pair for the run generators X, Y, Z, |1><1|.
// complex128: in FP64.  complex64: the pair's value is formed in FP32 with FMAs
// (two roundings at most) and returned as a double; the sums over pairs, warps,
// tiles and the state are FP64.
template <typename R, int CODE>
__device__ __forceinline__ double pair_gen_im_k(C<R> a0, C<R> a1, C<R> b0, C<R> b1) {
    // w = G a;  Im(conj(b) w) = b.x w.y - b.y w.x
    R r;
    if constexpr (CODE == 1) r = fma(b0.x, a1.y, -(b0.y * a1.x)) + fma(b1.x, a0.y, -(b1.y * a0.x));  // w = (a1, a0)
    else if constexpr (CODE == 2) r = fma(b1.x, a0.x, b1.y * a0.y) - fma(b0.x, a1.x, b0.y * a1.y);   // w = (-i a1, i a0)
    else if constexpr (CODE == 3) r = fma(b0.x, a0.y, -(b0.y * a0.x)) - fma(b1.x, a1.y, -(b1.y * a1.x));  // (a0, -a1)
    else r = fma(b1.x, a1.y, -(b1.y * a1.x));                                                          // w = (0, a1)
    return (double)r;
}
template <typename R>
__device__ __forceinline__ double pair_gen_im(int code, C<R> a0, C<R> a1, C<R> b0, C<R> b1) {
    switch (code) {
    case 1: return pair_gen_im_k<R, 1>(a0, a1, b0, b1);
    case 2: return pair_gen_im_k<R, 2>(a0, a1, b0, b1);
    case 3: return pair_gen_im_k<R, 3>(a0, a1, b0, b1);
    default: return pair_gen_im_k<R, 4>(a0, a1, b0, b1);
    }
}

// Run signature: length and, per member in application order, structure and generator
// code (0: no gradient).  The common signatures get pair loops with both known at compile
// time (no per-pair dispatch); the others use the run-time loops below.
__host__ __device__ constexpr int run_sig(int len, int k0, int g0, int k1 = 0, int g1 = 0, int k2 = 0, int g2 = 0) {
    return len | (k0 << 2) | (g0 << 5) | (k1 << 8) | (g1 << 11) | (k2 << 14) | (g2 << 17);
}

// forward pair loop: members applied one by one in their structured forms
template <typename R, int NS, int LEN, int K0, int K1, int K2>
__device__ __forceinline__ void run_fwd_fixed(C<R> *const (&s)[NS], const Range &rg, uint32_t low, uint32_t bit,
                                              const C<R> (&m)[kMaxRun][4]) {
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t i0 = ((g & ~low) << 1) | (g & low), i1 = i0 | bit;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            C<R> a0 = s[q][i0], a1 = s[q][i1];
            apply_pair_k<R, K0>(m[0], a0, a1);
            if constexpr (LEN > 1) apply_pair_k<R, K1>(m[1], a0, a1);
            if constexpr (LEN > 2) apply_pair_k<R, K2>(m[2], a0, a1);
            s[q][i0] = a0;
            s[q][i1] = a1;
        }
    }
}

// m0 v0 + m1 v1 with one rounding per FMA step (complex64: paired FP32 instructions)
template <typename R> __device__ __forceinline__ C<R> mac2(C<R> m0, C<R> v0, C<R> m1, C<R> v1);
template <> __device__ __forceinline__ float2 mac2<float>(float2 m0, float2 v0, float2 m1, float2 v1) {
    const float2 t = cmul2(m0, v0);
    const float2 w = __ffma2_rn(make_float2(m1.y, m1.y), make_float2(-v1.y, v1.x), t);
    return __ffma2_rn(make_float2(m1.x, m1.x), v1, w);
}
template <> __device__ __forceinline__ double2 mac2<double>(double2 m0, double2 v0, double2 m1, double2 v1) {
    CAcc<double> a;
    a.set(m0, v0);
    a.add(m1, v1);
    return a.get();
}

// Adjoint sweep over a run, fused.  With A_k the product of the inverses undone before member k
// (reverse order, A_0 = I), member k's generator product at its point of the sweep is
// Im(b^dagger H_k a) on the run's input pair (a of lambda, b of the bra), H_k = A_k^dagger G_k A_k
// Hermitian: h00 Im(b0* a0) + h11 Im(b1* a1) + Re h01 (Im(b0* a1) + Im(b1* a0))
// + Im h01 (Re(b0* a1) - Re(b1* a0)).  The four cross terms are formed once per pair, each member
// adds one FMA chain, and the run's inverse (the product of its members' inverses) is applied
// to both states as one 2x2 (FMA chains, as the structured members of the forward runs).  H_k and the product are formed in FP64 per
// segment (fuse_rev_run).
template <typename R, int NS, int LEN, bool ALLG>
__device__ __forceinline__ void run_rev_fused(C<R> *const (&s)[NS], const Range &rg, uint32_t low, uint32_t bit,
                                              const C<R> (&M)[4], const R (&h)[kMaxRun][4],
                                              const bool (&has)[kMaxRun], double (&ip)[kMaxRun]) {
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t i0 = ((g & ~low) << 1) | (g & low), i1 = i0 | bit;
        const C<R> a0 = s[0][i0], a1 = s[0][i1], b0 = s[NS - 1][i0], b1 = s[NS - 1][i1];
        const R x1 = fma(b0.x, a0.y, -(b0.y * a0.x));
        const R x2 = fma(b1.x, a1.y, -(b1.y * a1.x));
        const R s1 = fma(b0.x, a1.y, -(b0.y * a1.x)) + fma(b1.x, a0.y, -(b1.y * a0.x));
        const R s2 = fma(b0.x, a1.x, b0.y * a1.y) - fma(b1.x, a0.x, b1.y * a0.y);
#pragma unroll
        for (int k = 0; k < LEN; ++k)
            if (ALLG || has[k]) ip[k] += (double)fma(h[k][0], x1, fma(h[k][1], x2, fma(h[k][2], s1, h[k][3] * s2)));
        s[0][i0] = mac2<R>(M[0], a0, M[1], a1);
        s[0][i1] = mac2<R>(M[2], a0, M[3], a1);
        s[NS - 1][i0] = mac2<R>(M[0], b0, M[1], b1);
        s[NS - 1][i1] = mac2<R>(M[2], b0, M[3], b1);
    }
}

// Replace the adjoint coefficients of a run (slots cf[0..len-1], staged for the reverse sweep)
// by its fused form: cf[0] the product of the members' inverses; cf[1] = (h00, h11), h01 of
// members 0 and 1 of the sweep, cf[2] the same for member 2.  FP64 from the staged coefficients.
template <typename R>
__device__ void fuse_rev_run(const DOp *ops, C<R> (*cf)[4], int len) {
    auto mul = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
    auto cj = [](double2 a) { return make_double2(a.x, -a.y); };
    // member matrices (adjoints, sweep order), read before cf is overwritten
    double2 m[kMaxRun][4];
#pragma unroll
    for (int k = 0; k < kMaxRun; ++k) {
        if (k < len) {
            C<R> t[4];
            member_from<R>(ops[len - 1 - k], cf[len - 1 - k], t);
#pragma unroll
            for (int i = 0; i < 4; ++i) m[k][i] = make_double2((double)t[i].x, (double)t[i].y);
        }
    }
    double2 A[4] = {make_double2(1, 0), make_double2(0, 0), make_double2(0, 0), make_double2(1, 0)};
    double hv[kMaxRun][4];
#pragma unroll
    for (int k = 0; k < kMaxRun; ++k) {
        hv[k][0] = hv[k][1] = hv[k][2] = hv[k][3] = 0.0;
        if (k >= len) continue;
        const DOp &op = ops[len - 1 - k];
        const int code = op.gslot >= 0 ? op.gcode : 0;
        if (code) {
            const double2 z = make_double2(0, 0), one = make_double2(1, 0);
            double2 G[4];
            if (code == 1) { G[0] = z; G[1] = one; G[2] = one; G[3] = z; }
            else if (code == 2) { G[0] = z; G[1] = make_double2(0, -1); G[2] = make_double2(0, 1); G[3] = z; }
            else if (code == 3) { G[0] = one; G[1] = z; G[2] = z; G[3] = make_double2(-1, 0); }
            else { G[0] = z; G[1] = z; G[2] = z; G[3] = one; }
            double2 GA[4];
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int c = 0; c < 2; ++c) GA[r * 2 + c] = add(mul(G[r * 2], A[c]), mul(G[r * 2 + 1], A[2 + c]));
            // H = A^dagger (G A): h00, h11 and h01
            hv[k][0] = add(mul(cj(A[0]), GA[0]), mul(cj(A[2]), GA[2])).x;
            hv[k][1] = add(mul(cj(A[1]), GA[1]), mul(cj(A[3]), GA[3])).x;
            const double2 h01 = add(mul(cj(A[0]), GA[1]), mul(cj(A[2]), GA[3]));
            hv[k][2] = h01.x;
            hv[k][3] = h01.y;
        }
        double2 B[4];
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) B[r * 2 + c] = add(mul(m[k][r * 2], A[c]), mul(m[k][r * 2 + 1], A[2 + c]));
#pragma unroll
        for (int i = 0; i < 4; ++i) A[i] = B[i];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) cf[0][i] = mk<R>((R)A[i].x, (R)A[i].y);
    cf[1][0] = mk<R>((R)hv[0][0], (R)hv[0][1]);
    cf[1][1] = mk<R>((R)hv[0][2], (R)hv[0][3]);
    cf[1][2] = mk<R>((R)hv[1][0], (R)hv[1][1]);
    cf[1][3] = mk<R>((R)hv[1][2], (R)hv[1][3]);
    if (len > 2) {
        cf[2][0] = mk<R>((R)hv[2][0], (R)hv[2][1]);
        cf[2][1] = mk<R>((R)hv[2][2], (R)hv[2][3]);
    }
}

// A run of `len` single-wire gates on bit rb, applied per amplitude pair in registers.
// Forward: structured members are applied one by one; a run with a general member has its
// product formed once in FP64 and applied as one 2x2 matrix.
// Adjoint: the members are undone one by one with the generator products between them.
template <typename R, int NS, bool REV>
__device__ void exec_run(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp *__restrict__ ops,
                         const C<R> (*cf)[4], int len,
                         const double4 *__restrict__ cs, const double2 *__restrict__ consts, double *gradw,
                         bool first_tile) {
    const int rb = ops[0].rbit;
    const uint32_t low = (1u << rb) - 1;
    const uint32_t bit = 1u << rb;
    const Range rg = groups(kt, wl, 1, wloc);
    if (!REV) {
        // structured members (no general 2x2 among them) are cheaper one by one than their
        // product, which is a general 2x2
        C<R> mm[kMaxRun][4];
        int kinds[kMaxRun];
        bool all_structured = true;
#pragma unroll
        for (int k = 0; k < kMaxRun; ++k) {
            kinds[k] = MK_GENERAL;
            if (k < len) {
                member_from<R>(ops[k], cf[k], mm[k]);
                kinds[k] = ops[k].mkind;
                all_structured = all_structured && kinds[k] != MK_GENERAL;
            }
        }
        if (all_structured) {
            switch (run_sig(len, kinds[0], 0, kinds[1], 0, kinds[2], 0)) {
            case run_sig(3, MK_DIAG, 0, MK_REAL, 0, MK_DIAG, 0):
                run_fwd_fixed<R, NS, 3, MK_DIAG, MK_REAL, MK_DIAG>(s, rg, low, bit, mm);
                return;
            case run_sig(2, MK_REAL, 0, MK_DIAG, 0):
                run_fwd_fixed<R, NS, 2, MK_REAL, MK_DIAG, MK_GENERAL>(s, rg, low, bit, mm);
                return;
            case run_sig(2, MK_DIAG, 0, MK_REAL, 0):
                run_fwd_fixed<R, NS, 2, MK_DIAG, MK_REAL, MK_GENERAL>(s, rg, low, bit, mm);
                return;
            default:
                for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
                    const uint32_t i0 = ((g & ~low) << 1) | (g & low), i1 = i0 | bit;
#pragma unroll
                    for (int q = 0; q < NS; ++q) {
                        C<R> a0 = s[q][i0], a1 = s[q][i1];
#pragma unroll
                        for (int k = 0; k < kMaxRun; ++k)
                            if (k < len) apply_pair<R>(kinds[k], mm[k], a0, a1);
                        s[q][i0] = a0;
                        s[q][i1] = a1;
                    }
                }
                return;
            }
        }
        // product M = m_{len-1} ... m_0 in FP64
        double2 P[4] = {make_double2(1, 0), make_double2(0, 0), make_double2(0, 0), make_double2(1, 0)};
        for (int k = 0; k < len; ++k) {
            C<double> q[4];
            member_mat<double>(ops[k], cs, consts, false, q);
            double2 Q[4];
            for (int r = 0; r < 2; ++r)
                for (int c = 0; c < 2; ++c) {
                    const double2 x0 = q[r * 2 + 0], x1 = q[r * 2 + 1], y0 = P[0 * 2 + c], y1 = P[1 * 2 + c];
                    Q[r * 2 + c] = make_double2(x0.x * y0.x - x0.y * y0.y + x1.x * y1.x - x1.y * y1.y,
                                                x0.x * y0.y + x0.y * y0.x + x1.x * y1.y + x1.y * y1.x);
                }
            P[0] = Q[0]; P[1] = Q[1]; P[2] = Q[2]; P[3] = Q[3];
        }
        C<R> m[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) m[i] = mk<R>((R)P[i].x, (R)P[i].y);
        for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
            const uint32_t i0 = ((g & ~low) << 1) | (g & low), i1 = i0 | bit;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                const C<R> a0 = s[q][i0], a1 = s[q][i1];
                CAcc<R> p, r;
                p.set(m[0], a0); p.add(m[1], a1);
                r.set(m[2], a0); r.add(m[3], a1);
                s[q][i0] = p.get();
                s[q][i1] = r.get();
            }
        }
        return;
    }
    if constexpr (REV) {
        // adjoint sweep, fused per pair (run_rev_fused; coefficients from fuse_rev_run)
        C<R> M[4];
        R h[kMaxRun][4];
        bool has[kMaxRun];
        double ip[kMaxRun];
        int gc[kMaxRun];
#pragma unroll
        for (int i = 0; i < 4; ++i) M[i] = cf[0][i];
        h[0][0] = cf[1][0].x; h[0][1] = cf[1][0].y; h[0][2] = cf[1][1].x; h[0][3] = cf[1][1].y;
        h[1][0] = cf[1][2].x; h[1][1] = cf[1][2].y; h[1][2] = cf[1][3].x; h[1][3] = cf[1][3].y;
        h[2][0] = h[2][1] = h[2][2] = h[2][3] = (R)0;
        if (len > 2) {
            h[2][0] = cf[2][0].x; h[2][1] = cf[2][0].y; h[2][2] = cf[2][1].x; h[2][3] = cf[2][1].y;
        }
        bool all = true;
#pragma unroll
        for (int kk = 0; kk < kMaxRun; ++kk) {
            ip[kk] = 0.0;
            gc[kk] = 0;
            if (kk < len) {
                const DOp &op = ops[len - 1 - kk];
                if (op.gslot >= 0) gc[kk] = op.gcode;
            }
            has[kk] = gc[kk] != 0;
            all = all && (kk >= len || has[kk]);
        }
        if (len == 3) {
            if (all) run_rev_fused<R, NS, 3, true>(s, rg, low, bit, M, h, has, ip);
            else run_rev_fused<R, NS, 3, false>(s, rg, low, bit, M, h, has, ip);
        } else {
            if (all) run_rev_fused<R, NS, 2, true>(s, rg, low, bit, M, h, has, ip);
            else run_rev_fused<R, NS, 2, false>(s, rg, low, bit, M, h, has, ip);
        }
#pragma unroll
        for (int kk = 0; kk < kMaxRun; ++kk)
            if (kk < len && gc[kk]) add_grad(gradw, ops[len - 1 - kk].gslot, ip[kk], first_tile);

    }
}

// ---- two runs on different bits in one pass over amplitude quadruples -------------------
// Forward sweeps apply consecutive runs A on bit a and B on bit b per quadruple
// {i, i|a, i|b, i|a|b}: A on the pairs along a, then B on the pairs along b.  Every amplitude
// sees the same operations in the same order as with two separate passes (results are
// bit-identical), while the tile is read and written once instead of twice, addressed once
// and synchronised once: 73.8 vs 76.7 ms for the 1024-circuit forward + VJP step, 5 % on
// the HEA forward batch.  The adjoint sweep keeps one run per pass: pairing it as well
// (generator products over both pairs of a quadruple between the undone members) measured
// slower, 77.9 ms, as the quadruples of two states and six products do not fit the
// registers left.

// Forward run signatures that pair; DOp::pair of a run head holds the code (1..3) of the
// pairing with the next run in op order, chosen on the host (mark_pairs).
__host__ __device__ constexpr int pair_sig(int code) {
    return code == 1 ? run_sig(3, MK_DIAG, 0, MK_REAL, 0, MK_DIAG, 0)
           : code == 2 ? run_sig(2, MK_REAL, 0, MK_DIAG, 0)
                       : run_sig(2, MK_DIAG, 0, MK_REAL, 0);
}

struct Quad {
    uint32_t lowp, lowq, ba, bb;  // insertion masks of the lower / higher bit; bits of runs A and B
    __device__ __forceinline__ uint32_t base(uint32_t g) const {
        const uint32_t x = ((g & ~lowp) << 1) | (g & lowp);
        return ((x & ~lowq) << 1) | (x & lowq);
    }
};

template <typename R, int LEN, int K0, int K1, int K2>
__device__ __forceinline__ void run_members(const C<R> (&m)[kMaxRun][4], C<R> &v0, C<R> &v1) {
    apply_pair_k<R, K0>(m[0], v0, v1);
    if constexpr (LEN > 1) apply_pair_k<R, K1>(m[1], v0, v1);
    if constexpr (LEN > 2) apply_pair_k<R, K2>(m[2], v0, v1);
}

template <typename R, int NS, int LEN, int K0, int K1, int K2>
__device__ __forceinline__ void run2_fwd_fixed(C<R> *const (&s)[NS], const Range &rg, const Quad &qd,
                                               const C<R> (&ma)[kMaxRun][4], const C<R> (&mb)[kMaxRun][4]) {
    for (uint32_t g = rg.g0; g < rg.g1; g += rg.gs) {
        const uint32_t i0 = qd.base(g), i1 = i0 | qd.ba, i2 = i0 | qd.bb, i3 = i1 | qd.bb;
#pragma unroll
        for (int q = 0; q < NS; ++q) {
            C<R> v0 = s[q][i0], v1 = s[q][i1], v2 = s[q][i2], v3 = s[q][i3];
            run_members<R, LEN, K0, K1, K2>(ma, v0, v1);
            run_members<R, LEN, K0, K1, K2>(ma, v2, v3);
            run_members<R, LEN, K0, K1, K2>(mb, v0, v2);
            run_members<R, LEN, K0, K1, K2>(mb, v1, v3);
            s[q][i0] = v0;
            s[q][i1] = v1;
            s[q][i2] = v2;
            s[q][i3] = v3;
        }
    }
}

// Runs A (ops opa, first in op order) and B (opb) of equal pairable signature `sig`.
template <typename R, int NS>
__device__ __forceinline__ void exec_run2(C<R> *const (&s)[NS], int kt, int wl, bool wloc, const DOp *__restrict__ opa,
                                       const C<R> (*cfa)[4], const DOp *__restrict__ opb, const C<R> (*cfb)[4],
                                       int len, int sig) {
    C<R> ma[kMaxRun][4], mb[kMaxRun][4];
#pragma unroll
    for (int k = 0; k < kMaxRun; ++k) {
        if (k < len) {
            member_from<R>(opa[k], cfa[k], ma[k]);
            member_from<R>(opb[k], cfb[k], mb[k]);
        }
    }
    Quad qd;
    qd.ba = 1u << opa[0].rbit;
    qd.bb = 1u << opb[0].rbit;
    const int p = min((int)opa[0].rbit, (int)opb[0].rbit), q = max((int)opa[0].rbit, (int)opb[0].rbit);
    qd.lowp = (1u << p) - 1;
    qd.lowq = (1u << q) - 1;
    const Range rg = groups(kt, wl, 2, wloc);
    switch (sig) {
    case run_sig(3, MK_DIAG, 0, MK_REAL, 0, MK_DIAG, 0):
        run2_fwd_fixed<R, NS, 3, MK_DIAG, MK_REAL, MK_DIAG>(s, rg, qd, ma, mb);
        break;
    case run_sig(2, MK_REAL, 0, MK_DIAG, 0):
        run2_fwd_fixed<R, NS, 2, MK_REAL, MK_DIAG, MK_GENERAL>(s, rg, qd, ma, mb);
        break;
    default:
        run2_fwd_fixed<R, NS, 2, MK_DIAG, MK_REAL, MK_GENERAL>(s, rg, qd, ma, mb);
        break;
    }
}

__device__ __forceinline__ uint64_t insert_zeros64(uint64_t v, const uint8_t *bits, int nb) {
    for (int j = 0; j < nb; ++j) {
        const uint64_t lo = v & ((uint64_t(1) << bits[j]) - 1);
        v = ((v ^ lo) << 1) | lo;
    }
    return v;
}

// sum_t coeff_t <psi|P_t|psi> per observable into acc[obs] (per-thread part)
template <typename R>
__device__ void expval_terms(const C<R> *psi, uint64_t n_amp, const DTerm *__restrict__ terms, uint32_t nterms,
                             uint32_t obs0, double (&acc)[kObsPerPass]) {
    // observables obs0 .. obs0 + kObsPerPass - 1 of the circuit (accumulator o <-> obs0 + o)
    for (uint32_t t = 0; t < nterms; ++t) {
        DTerm tm = terms[t];
        if (tm.obs < obs0 || tm.obs >= obs0 + kObsPerPass) continue;
        tm.obs -= obs0;
        double a = 0.0;
        if (tm.xmask == 0) {  // diagonal word (ny is 0): sum of +-|psi_i|^2, one read per amplitude
            for (uint64_t i = threadIdx.x; i < n_amp; i += blockDim.x) {
                const double2 v = widen<R>(psi[i]);
                const double p = v.x * v.x + v.y * v.y;
                a += (__popcll(i & tm.zmask) & 1) ? -p : p;
            }
#pragma unroll
            for (int o = 0; o < kObsPerPass; ++o)
                if (o == (int)tm.obs) acc[o] += tm.coeff * a;
            continue;
        }
        for (uint64_t i = threadIdx.x; i < n_amp; i += blockDim.x) {
            // Re conj(psi_{i^X}) i^ny (-1)^{|i&Z|} psi_i
            const double2 vi = widen<R>(psi[i]), vj = widen<R>(psi[i ^ tm.xmask]);
            const double zr = vj.x * vi.x + vj.y * vi.y, zi = vj.x * vi.y - vj.y * vi.x;
            double r;
            switch (tm.ny & 3) {
            case 0: r = zr; break;
            case 1: r = -zi; break;
            case 2: r = -zr; break;
            default: r = zi; break;
            }
            a += (__popcll(i & tm.zmask) & 1) ? -r : r;
        }
#pragma unroll
        for (int o = 0; o < kObsPerPass; ++o)  // constant indices keep acc in registers
            if (o == (int)tm.obs) acc[o] += tm.coeff * a;
    }
}

// bra_j = sum_t w_t (P_t psi)_j,  (P psi)_j = i^ny (-1)^{|(j^X)&Z|} psi_{j^X}
template <typename R>
__device__ void init_bra(C<R> *bra, const C<R> *psi, uint64_t n_amp, const DTerm *__restrict__ terms,
                         uint32_t nterms, const double *__restrict__ dy, bool weighted) {
    for (uint64_t j = threadIdx.x; j < n_amp; j += blockDim.x) {
        double br = 0.0, bi = 0.0;
        double fd = 0.0;  // diagonal words: bra_j gets (sum of +-w) * psi_j, psi_j read once
        for (uint32_t t = 0; t < nterms; ++t) {
            const DTerm tm = terms[t];
            const double w = weighted ? tm.coeff : tm.coeff * dy[tm.obs];
            if (w == 0.0) continue;
            if (tm.xmask == 0 && (tm.ny & 3) == 0) {
                fd += (__popcll(j & tm.zmask) & 1) ? -w : w;
                continue;
            }
            const uint64_t i = j ^ tm.xmask;
            const double2 v = widen<R>(psi[i]);
            double fr = (__popcll(i & tm.zmask) & 1) ? -w : w, fi = 0.0;
            switch (tm.ny & 3) {
            case 1: fi = fr; fr = 0; break;
            case 2: fr = -fr; break;
            case 3: fi = -fr; fr = 0; break;
            default: break;
            }
            br += fr * v.x - fi * v.y;
            bi += fr * v.y + fi * v.x;
        }
        if (fd != 0.0) {
            const double2 v = widen<R>(psi[j]);
            br += fd * v.x;
            bi += fd * v.y;
        }
        bra[j] = mk<R>((R)br, (R)bi);
    }
}

struct KArgs {
    const DCirc *circs;
    const DSeg *segs;
    const DOp *ops;
    const DTerm *terms;
    const double2 *consts;
    const uint32_t *order;
    uint32_t ncirc;
    uint32_t *counter;
    const double4 *cs;    // per-parameter trigonometry
    const double *dy;     // [sum nobs] (VJP)
    double *out;          // forward: [sum nobs]
    double *gradw;        // VJP: [ngslots * nwarps]
    void *pool_a, *pool_b;
    const int *reuse;     // VJP: nonzero when pool A still holds this step's forward states
    const void *rcf;      // VJP: per op, the reverse sweep's coefficients (k_rev_coeffs)
    int max_kt;
};

template <typename R> __device__ __forceinline__ void zero_tile(C<R> *s, uint32_t n) {
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s[i] = mk<R>(0, 0);
}

// Tile element l lives at tbase | deposit(l over lbits).  Threads take l = tid + k*blockDim
// (blockDim a power of two), so the deposit of the low bits is fixed per thread and
// only the few high bits change with k.
__device__ __forceinline__ uint64_t deposit_bits(uint32_t v, const uint8_t *bits, int from, int to) {
    uint64_t r = 0;
    for (int j = from; j < to; ++j)
        if (v & (1u << (j - from))) r |= uint64_t(1) << bits[j];
    return r;
}
template <typename R, bool LOAD>
__device__ __forceinline__ void move_tile(C<R> *sm, C<R> *gm, const DSeg &sg, uint64_t tbase, uint32_t nt) {
    const int bl = 31 - __clz((int)blockDim.x);
    // 16-byte chunks of V consecutive amplitudes, contiguous in both memories when the tile
    // holds state bit 0 (the planner keeps the lowest state bits in every tile).  The thread's
    // bits are deposited once; a chunk's higher bits are an OR of precomputed masks.
    constexpr int LV = sizeof(C<R>) == 8 ? 1 : 0;
    const int hb0 = LV + bl;
    if ((LV == 0 || sg.lbits[0] == 0) && (nt >> LV) >= blockDim.x && sg.nl - hb0 <= 6) {
        const uint64_t lo = tbase | deposit_bits(threadIdx.x << LV, sg.lbits, 0, hb0);
        uint64_t hm[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) hm[i] = hb0 + i < sg.nl ? uint64_t(1) << sg.lbits[hb0 + i] : 0;
        const uint32_t per = (nt >> LV) >> bl;
        for (uint32_t j = 0; j < per; ++j) {
            uint64_t hi = 0;
#pragma unroll
            for (int i = 0; i < 6; ++i)
                if ((j >> i) & 1u) hi |= hm[i];
            float4 *g4 = reinterpret_cast<float4 *>(gm + (lo | hi));
            float4 *s4 = reinterpret_cast<float4 *>(sm + ((threadIdx.x + (j << bl)) << LV));
            if (LOAD) {
                // straight to shared memory: every chunk of the tile is in flight at once
                const unsigned sa = (unsigned)__cvta_generic_to_shared(s4);
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g4) : "memory");
            } else {
                *g4 = *s4;
            }
        }
        return;  // loads: the caller waits (tile_wait) and then synchronises
    }
    if (nt <= blockDim.x) {
        if (threadIdx.x < nt) {
            const uint64_t a = tbase | deposit_bits(threadIdx.x, sg.lbits, 0, sg.nl);
            if (LOAD) sm[threadIdx.x] = gm[a];
            else gm[a] = sm[threadIdx.x];
        }
        return;
    }
    const uint64_t lo = tbase | deposit_bits(threadIdx.x, sg.lbits, 0, bl);
    for (uint32_t k = 0, l = threadIdx.x; l < nt; ++k, l += blockDim.x) {
        const uint64_t a = lo | deposit_bits(k, sg.lbits, bl, sg.nl);
        if (LOAD) sm[l] = gm[a];
        else gm[a] = sm[l];
    }
}
// completes this thread's tile loads (cp.async); a barrier must follow before other threads read
__device__ __forceinline__ void tile_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
template <typename R>
__device__ void load_tile(C<R> *dst, const C<R> *__restrict__ src, const DSeg &sg, uint64_t tbase, uint32_t nt) {
    move_tile<R, true>(dst, const_cast<C<R> *>(src), sg, tbase, nt);
}
template <typename R>
__device__ void store_tile(C<R> *__restrict__ dst, const C<R> *src, const DSeg &sg, uint64_t tbase, uint32_t nt) {
    move_tile<R, false>(const_cast<C<R> *>(src), dst, sg, tbase, nt);
}

// Apply the gates of one segment to the tile(s): forward (NS = 1) or the adjoint
// sweep over (lambda, bra) with gradient products (NS = 2, REV).
template <typename R, int NS, bool REV, bool FULL>
__device__ void exec_segment(const KArgs &A, C<R> *const (&tiles)[NS], int kt, const DSeg &sg, const DOp *ops,
                             const C<R> (*cf)[4], bool first_tile) {
    const int wl = kt - (31 - __clz((int)(blockDim.x >> 5)));  // bits owned by one warp's block
    bool prev_wloc = false;
    int o = REV ? (int)sg.nops - 1 : 0;
    while (REV ? o >= 0 : o < (int)sg.nops) {
        // find the step: a fused run (head op carries run >= 2) or a single gate
        int head = o, len = 1;
        if (REV) {
            // the sweep meets runs at their last member, which points back to the head
            const int h = o - ops[o].back;
            if (h != o) {
                head = h;
                len = ops[h].run;
            }
        } else {
            const DOp &hd = ops[o];
            if (hd.run >= 2) len = hd.run;
        }
        const DOp *op0 = ops + head;
        // forward: a run paired on the host with the next run (same signature, other bit)
        int head2 = -1, sig = 0;
        if (!REV && len >= 2 && op0->pair != 0) {
            head2 = head + len;
            sig = pair_sig(op0->pair);
        }
        const bool wloc = head2 >= 0 ? wl >= 2 && op0->maxbit < wl && ops[head2].maxbit < wl
                                     : wl >= 1 && op0->maxbit < wl && (len >= 2 || op0->nb <= wl);
        if (prev_wloc && wloc) __syncwarp();
        else __syncthreads();
        if (head2 >= 0) {
            exec_run2<R, NS>(tiles, kt, wl, wloc, op0, cf + head, ops + head2, cf + head2, len, sig);
            prev_wloc = wloc;
            o = head2 + len;
            continue;
        }
        if (len >= 2) {
            exec_run<R, NS, REV>(tiles, kt, wl, wloc, op0, cf + head, len, A.cs, A.consts, A.gradw, first_tile);
        } else {
            const DOp op = *op0;
            if (REV && op.gslot >= 0) {
                add_grad(A.gradw, op.gslot, gen_inner<R, FULL>(tiles[NS - 1], tiles[0], kt, wl, wloc, op, A.consts),
                         first_tile);
                if (wloc) __syncwarp();
                else __syncthreads();
            }
            if constexpr (FULL) {
                if (op.form == F_MATK) {
                    apply_matk<R, NS>(tiles, kt, wl, wloc, op, A.consts, REV);
                } else {
                    C<R> m[16];
                    op_coeffs<R, 16>(op, A.cs, A.consts, REV, m);
                    apply_op_general<R, NS>(tiles, kt, wl, wloc, op, m);
                }
            } else {
                C<R> m[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) m[r] = cf[head][r];
                apply_op<R, NS>(tiles, kt, wl, wloc, op, m);
            }
        }
        prev_wloc = wloc;
        o = REV ? head - 1 : head + len;
    }
    __syncthreads();
}

// Stage segment `idx` in shared memory: its bit tables are indexed by loop variables in the
// tile moves, which would put a register copy of the record in local memory.
// Its op records go to shared memory too, with each op's coefficients (forward or adjoint,
// `adj`) computed once per segment instead of by every thread at every step of every tile.
template <typename R>
__device__ __forceinline__ const DSeg &stage_segment(DSeg *s_seg, DOp *s_ops, C<R> (*s_cf)[4], const KArgs &A,
                                                     uint32_t idx, bool adj) {
    __syncthreads();
    if (threadIdx.x < sizeof(DSeg) / 4)
        reinterpret_cast<uint32_t *>(s_seg)[threadIdx.x] = reinterpret_cast<const uint32_t *>(A.segs + idx)[threadIdx.x];
    const DSeg &g = A.segs[idx];
    const uint32_t words = g.nops * (uint32_t)(sizeof(DOp) / 4);
    const uint32_t *src = reinterpret_cast<const uint32_t *>(A.ops + g.op_begin);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) reinterpret_cast<uint32_t *>(s_ops)[i] = src[i];
    if (adj) {  // the reverse sweep's coefficients, formed once per launch by k_rev_coeffs
        const C<R> *src = static_cast<const C<R> *>(A.rcf) + (size_t)g.op_begin * 4;
        for (uint32_t i = threadIdx.x; i < g.nops * 4; i += blockDim.x) (&s_cf[0][0])[i] = src[i];
    } else {
        for (uint32_t o = threadIdx.x; o < g.nops; o += blockDim.x) {
            const DOp &op = A.ops[g.op_begin + o];
            if (op.form == F_MAT2 || op.form == F_PAIR4 || op.form == F_MATK) continue;  // formed where they are used
            C<R> t[4];
            op_coeffs<R, 4>(op, A.cs, A.consts, adj, t);
#pragma unroll
            for (int r = 0; r < 4; ++r) s_cf[o][r] = t[r];
        }
    }
    __syncthreads();
    return *s_seg;
}

// Stage a circuit's observable terms in shared memory (the op-record buffer, free between
// segments) when they fit; with dy given, each coefficient is multiplied by its output's dy.
// Returns where the terms are to be read.
__device__ __forceinline__ const DTerm *stage_terms(DTerm *s_terms, const KArgs &A, const DCirc &c,
                                                    const double *dy) {
    const DTerm *g = A.terms + c.term_begin;
    if (c.nterms > kMaxSegOpsStaged * sizeof(DOp) / sizeof(DTerm)) return g;
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < c.nterms; t += blockDim.x) {
        DTerm x = g[t];
        if (dy) x.coeff *= dy[x.obs];
        s_terms[t] = x;
    }
    __syncthreads();
    return s_terms;
}

// one circuit, forward: state ends in tile 0 (resident) or pool A (global)
template <typename R, bool FULL>
__device__ void run_forward(const KArgs &A, const DCirc &c, C<R> *sm, C<R> *pa, DSeg *s_seg, DOp *s_ops,
                            C<R> (*s_cf)[4]) {
    const uint32_t tn = 1u << c.kt;
    C<R> *tiles[1] = {sm};
    if (c.resident) {
        zero_tile<R>(sm, tn);
        __syncthreads();
        if (threadIdx.x == 0) sm[0] = mk<R>(1, 0);
        for (uint32_t si = 0; si < c.nseg; ++si) {
            const DSeg &sg = stage_segment<R>(s_seg, s_ops, s_cf, A, c.seg_begin + si, false);
            exec_segment<R, 1, false, FULL>(A, tiles, c.kt, sg, s_ops, s_cf, true);
        }
        return;
    }
    const uint64_t ntiles = uint64_t(1) << (c.n - c.kt);
    for (uint32_t si = 0; si < c.nseg; ++si) {
        const DSeg &sg = stage_segment<R>(s_seg, s_ops, s_cf, A, c.seg_begin + si, false);
        for (uint64_t t = 0; t < ntiles; ++t) {
            const uint64_t tbase = insert_zeros64(t, sg.lbits, sg.nl);
            if (si == 0) {
                zero_tile<R>(sm, tn);
                __syncthreads();
                if (threadIdx.x == 0 && tbase == 0) sm[0] = mk<R>(1, 0);
            } else {
                load_tile<R>(sm, pa, sg, tbase, tn);
                tile_wait();
            }
            exec_segment<R, 1, false, FULL>(A, tiles, c.kt, sg, s_ops, s_cf, true);
            store_tile<R>(pa, sm, sg, tbase, tn);
            __syncthreads();
        }
    }
}

// The reverse sweep's coefficients of every op, once per VJP launch (after k_trig): the
// adjoint coefficients of single ops and, for a run of single-wire gates, the fused form of
// fuse_rev_run in the run's slots.  Two-wire dense, double-excitation and k-wire matrix steps
// form theirs where they are used.  Kept out of k_batch, whose registers it would otherwise
// share.
template <typename R>
__global__ void k_rev_coeffs(const DOp *__restrict__ ops, uint32_t nops, const double4 *__restrict__ cs,
                             const double2 *__restrict__ consts, C<R> (*rcf)[4]) {
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < nops; o += gridDim.x * blockDim.x) {
        const DOp &op = ops[o];
        if (op.back != 0) continue;  // a run member: written by its run's head
        if (op.form == F_MAT2 || op.form == F_PAIR4 || op.form == F_MATK) continue;
        const int len = op.run >= 2 ? op.run : 1;
        for (int k = 0; k < len; ++k) {
            C<R> t[4];
            op_coeffs<R, 4>(ops[o + k], cs, consts, true, t);
            for (int r = 0; r < 4; ++r) rcf[o + k][r] = t[r];
        }
        if (len >= 2) fuse_rev_run<R>(ops + o, rcf + o, len);
    }
}

// MODE 0: forward expectation values; MODE 1: forward (unless reused) and the VJP sweep.
// FULL: compiled with the two-wire dense step and generator paths (only batches that
// hold such gates launch it; the others get a kernel without them, in fewer registers).
// Compiled for 512 threads (128 registers a thread).  Instantiations for 256 threads with up to
// 255 registers (no spills in the complex128 steps) were tried: the autotuner kept 512 threads
// for every workload of the bench (complex128 HEA batch 1027 ms either way).
template <typename R, int MODE, bool FULL>
__global__ void __launch_bounds__(512) k_batch(KArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint32_t s_next;
    __shared__ double s_red[kObsPerPass * 32];
    __shared__ __align__(8) DSeg s_seg;
    __shared__ __align__(8) DOp s_ops[kMaxSegOpsStaged];
    __shared__ __align__(16) C<R> s_cf[kMaxSegOpsStaged][4];
    C<R> *sm0 = reinterpret_cast<C<R> *>(smem_raw);
    C<R> *sm1 = sm0 + (size_t(1) << A.max_kt);
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(A.counter, 1u);
        __syncthreads();
        const uint32_t pos = s_next;
        __syncthreads();
        if (pos >= A.ncirc) break;
        const DCirc c = A.circs[A.order[pos]];
        C<R> *pa = static_cast<C<R> *>(A.pool_a) + c.off_a;
        C<R> *pb = static_cast<C<R> *>(A.pool_b) + c.off_b;
        const uint64_t namp = uint64_t(1) << c.n;
        const bool reuse = MODE == 1 && !c.resident && A.reuse && *A.reuse != 0;
        if (!reuse) run_forward<R, FULL>(A, c, sm0, pa, &s_seg, s_ops, s_cf);
        const C<R> *psi = c.resident ? sm0 : pa;
        if (MODE == 0) {
            const DTerm *T = stage_terms(reinterpret_cast<DTerm *>(s_ops), A, c, nullptr);
            // observables in groups of kObsPerPass, one group of accumulators at a time
            for (uint32_t obs0 = 0; obs0 < c.nobs; obs0 += kObsPerPass) {
                double acc[kObsPerPass];
#pragma unroll
                for (int o = 0; o < kObsPerPass; ++o) acc[o] = 0.0;
                expval_terms<R>(psi, namp, T, c.nterms, obs0, acc);
                block_reduce<kObsPerPass>(acc, s_red);
                if (threadIdx.x == 0) {
#pragma unroll
                    for (int o = 0; o < kObsPerPass; ++o)
                        if (obs0 + o < c.nobs) A.out[c.out_begin + obs0 + o] = acc[o];
                }
                __syncthreads();
            }
            continue;
        }
        // ---- VJP: bra = sum_o dy_o O_o psi, then the reverse sweep ----
        C<R> *bra = c.resident ? sm1 : pb;
        const DTerm *T = stage_terms(reinterpret_cast<DTerm *>(s_ops), A, c, A.dy + c.out_begin);
        init_bra<R>(bra, psi, namp, T, c.nterms, A.dy + c.out_begin, T != A.terms + c.term_begin);
        __syncthreads();
        C<R> *tiles[2] = {sm0, sm1};
        if (c.resident) {
            for (int32_t si = (int32_t)c.nseg - 1; si >= 0; --si) {
                const DSeg &sg = stage_segment<R>(&s_seg, s_ops, s_cf, A, c.seg_begin + si, true);
                exec_segment<R, 2, true, FULL>(A, tiles, c.kt, sg, s_ops, s_cf, true);
            }
            continue;
        }
        const uint64_t ntiles = uint64_t(1) << (c.n - c.kt);
        const uint32_t tn = 1u << c.kt;
        for (int32_t si = (int32_t)c.nseg - 1; si >= 0; --si) {
            const DSeg &sg = stage_segment<R>(&s_seg, s_ops, s_cf, A, c.seg_begin + si, true);
            for (uint64_t t = 0; t < ntiles; ++t) {
                const uint64_t tbase = insert_zeros64(t, sg.lbits, sg.nl);
                load_tile<R>(sm0, pa, sg, tbase, tn);
                load_tile<R>(sm1, pb, sg, tbase, tn);
                tile_wait();
                exec_segment<R, 2, true, FULL>(A, tiles, c.kt, sg, s_ops, s_cf, t == 0);
                store_tile<R>(pa, sm0, sg, tbase, tn);
                store_tile<R>(pb, sm1, sg, tbase, tn);
                __syncthreads();
            }
        }
    }
}

// flag <- valid && all(a == b)   (the caller copies `valid` into `flag` first)
__global__ void k_params_equal(const double *__restrict__ a, const double *__restrict__ b, uint64_t n, int *flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (a[i] != b[i]) *flag = 0;
}

// grad[p] = sum over ops referencing p (CSR order) of gscale * sum_w gradw[op, w]
__global__ void k_grad_params(const uint32_t *__restrict__ rowptr, const uint32_t *__restrict__ cols,
                              const double *__restrict__ gscale, const double *__restrict__ gradw, int nw,
                              uint64_t nparams, double *__restrict__ grad) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < nparams; p += (uint64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t k = rowptr[p]; k < rowptr[p + 1]; ++k) {
            const uint32_t g = cols[k];
            double v = 0.0;
            for (int w = 0; w < nw; ++w) v += gradw[(size_t)g * nw + w];
            s += gscale[g] * v;
        }
        grad[p] = s;
    }
}

// jac[jac_index[g]] = gscale * sum_w gradw[g, w]  (one observable pass)
__global__ void k_grad_scatter(const double *__restrict__ gscale, const double *__restrict__ gradw, int nw,
                               uint32_t ngslots, uint32_t obs, const uint32_t *__restrict__ gslot_circ,
                               const DCirc *__restrict__ circs, const uint64_t *__restrict__ jac_base,
                               const uint32_t *__restrict__ gslot_col, const uint32_t *__restrict__ circ_ncols,
                               double *__restrict__ jac) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngslots; g += gridDim.x * blockDim.x) {
        const uint32_t c = gslot_circ[g];
        if (obs >= circs[c].nobs) continue;
        double v = 0.0;
        for (int w = 0; w < nw; ++w) v += gradw[(size_t)g * nw + w];
        jac[jac_base[c] + (uint64_t)obs * circ_ncols[c] + gslot_col[g]] = gscale[g] * v;
    }
}

__global__ void k_onehot_dy(double *dy, const DCirc *circs, uint32_t ncirc, uint32_t obs) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncirc; c += gridDim.x * blockDim.x)
        for (uint32_t o = 0; o < circs[c].nobs; ++o) dy[circs[c].out_begin + o] = (o == obs) ? 1.0 : 0.0;
}

// ---------------------------------------------------------------------------
// host side
struct Config {
    int threads = 512;
    int kt = 13;
};

struct HostOp {
    uint32_t gate;
    std::vector<uint32_t> bits;  // circuit bit positions, gate order (controls first as in the reference)
    bool inv;
    int64_t pslot;
    std::vector<cd> cmat;  // constant matrix / phases (for constant gates)
    int form;
    int nt;                // number of targets (rest are controls)
    bool diff;             // differentiated (param op)
    int gen;               // generator id
};

struct Batch {
    int dtype = B200SV_C128;
    int device = 0;
    cudaStream_t own = nullptr, ext = nullptr;
    bool has_ext = false;  // set_stream called: ext (NULL = legacy default stream)
    cudaStream_t stream() const { return has_ext ? ext : own; }
    uint64_t nparams = 0;
    uint32_t ncirc = 0;
    Config cfg;
    bool use_graphs = false;
    bool full = false;  // the program holds two-wire dense steps or generators
    uint32_t last_launches = 0;

    // circuit descriptions kept for re-planning
    std::vector<uint32_t> nq;
    std::vector<std::vector<HostOp>> hops;
    std::vector<std::vector<DTerm>> hterms;  // masks in circuit bit positions
    std::vector<uint32_t> nobs;
    uint32_t total_obs = 0;

    // device program
    DCirc *d_circs = nullptr;
    DSeg *d_segs = nullptr;
    DOp *d_ops = nullptr;
    DTerm *d_terms = nullptr;
    double2 *d_consts = nullptr;
    uint32_t *d_order = nullptr;
    uint32_t *d_counter = nullptr;
    void *d_pool_a = nullptr, *d_pool_b = nullptr;
    size_t pool_a_bytes = 0, pool_b_bytes = 0;
    double *d_gradw = nullptr;
    double *d_gscale = nullptr;
    uint32_t *d_rowptr = nullptr, *d_cols = nullptr;
    uint32_t *d_gslot_circ = nullptr, *d_gslot_col = nullptr, *d_circ_ncols = nullptr;
    uint64_t *d_jac_base = nullptr;
    double *d_dy_tmp = nullptr;
    double *d_params_in = nullptr, *d_dy_in = nullptr, *d_out = nullptr, *d_grad = nullptr;
    double *d_params_fwd = nullptr;   // parameters of the last forward
    double4 *d_cs = nullptr;          // per-parameter trigonometry
    void *d_rcf = nullptr;            // per op: the reverse sweep's coefficients (k_rev_coeffs)
    uint32_t nops_total = 0;
    int *d_fwd_valid = nullptr;       // pool A holds the last forward's states
    int *d_reuse = nullptr;           // per-VJP decision
    uint32_t ngslots = 0;
    size_t smem_bytes = 0;
    int grid = 0;
    std::vector<DCirc> h_circs;
    std::vector<uint32_t> circ_ncols;
    std::vector<uint64_t> jac_base;
    uint64_t jac_total = 0;

    cudaGraphExec_t g_forward = nullptr, g_vjp = nullptr;

    std::vector<void *> allocs;
    ~Batch() {
        if (g_forward) cudaGraphExecDestroy(g_forward);
        if (g_vjp) cudaGraphExecDestroy(g_vjp);
        for (void *p : allocs) cudaFree(p);
        if (own) cudaStreamDestroy(own);
    }
    template <typename T> T *dalloc(size_t count) {
        void *p = nullptr;
        B200SV_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
        allocs.push_back(p);
        return static_cast<T *>(p);
    }
    void free_program() {
        if (g_forward) { cudaGraphExecDestroy(g_forward); g_forward = nullptr; }
        if (g_vjp) { cudaGraphExecDestroy(g_vjp); g_vjp = nullptr; }
        for (void *p : allocs) cudaFree(p);
        allocs.clear();
    }
    size_t amp() const { return dtype == B200SV_C64 ? 8 : 16; }
};

int popcount64(uint64_t x) { return __builtin_popcountll(x); }

// translate one reference operation into a batch op (circuit bit positions)
HostOp make_hostop(const b200sv_op &o, int64_t pslot, uint32_t nq, int dtype) {
    HostOp h{};
    h.gate = o.gate;
    h.inv = o.inverse != 0;
    h.pslot = pslot;
    h.diff = false;
    h.gen = -1;
    std::vector<uint32_t> w(o.wires, o.wires + o.nwires);
    check_wires(w.data(), (uint32_t)w.size(), nq, "batch op");
    std::vector<uint32_t> b(w.size());
    for (size_t i = 0; i < w.size(); ++i) b[i] = bitpos(w[i], nq);
    if (o.gate == B200SV_OP_MATRIX) {
        if (o.nwires < 1 || o.nwires > 4 || !o.matrix) throw Unsupported("batch: matrix ops act on 1 to 4 wires");
        const size_t d = size_t(1) << o.nwires;
        h.cmat.resize(d * d);
        for (size_t i = 0; i < d * d; ++i) {
            if (dtype == B200SV_C64) {
                const float *f = static_cast<const float *>(o.matrix);
                h.cmat[i] = cd(f[2 * i], f[2 * i + 1]);
            } else {
                const double *f = static_cast<const double *>(o.matrix);
                h.cmat[i] = cd(f[2 * i], f[2 * i + 1]);
            }
        }
        if (h.inv) h.cmat = dagger(h.cmat, d);
        h.gate = kConstGate;
        h.form = o.nwires == 1 ? F_MAT1 : o.nwires == 2 ? F_MAT2 : F_MATK;
        h.nt = (int)o.nwires;
        h.bits = b;
        return h;
    }
    if (o.gate >= kNumGates) throw ArgError("batch: unknown gate id");
    const GateInfo &gi = gate_table()[o.gate];
    if (gi.nwires >= 0 && (int)o.nwires != gi.nwires) throw ArgError(std::string("batch: wrong wire count for ") + gi.name);
    const bool param = gi.nparams == 1;
    if (gi.nparams > 1) throw Unsupported(std::string("batch: ") + gi.name + " must be decomposed into single-parameter gates");
    if (param && pslot < 0 && o.nparams != 1) throw ArgError(std::string("batch: ") + gi.name + " needs a parameter");
    h.bits = b;
    switch (o.gate) {
    case B200SV_Identity: h.form = F_NOOP; h.nt = 0; h.gate = kConstGate; return h;
    case B200SV_PauliX: h.form = F_SWAP; h.nt = 1; h.gate = kConstGate; return h;
    case B200SV_CNOT: h.form = F_SWAP; h.nt = 1; h.gate = kConstGate; return h;
    case B200SV_Toffoli: h.form = F_SWAP; h.nt = 1; h.gate = kConstGate; return h;
    case B200SV_SWAP: h.form = F_SWAP; h.nt = 2; h.gate = kConstGate; return h;
    case B200SV_CSWAP: h.form = F_SWAP; h.nt = 2; h.gate = kConstGate; return h;
    default: break;
    }
    // everything else: dense / diagonal, constant or parameterised
    auto constant = [&](int form, int nt, std::vector<cd> m) {
        h.form = form;
        h.nt = nt;
        h.gate = kConstGate;
        h.cmat = std::move(m);
        return h;
    };
    if (!param || pslot < 0) {
        // constant gate: reuse the plain-path compiler for the coefficients
        const double th = param ? o.params[0] : 0.0;
        GateDesc g = compile_gate(o.gate, o.wires, o.nwires, h.inv, param ? &th : nullptr, param ? 1 : 0, nq);
        switch (g.kind) {
        case Kind::Dense:
            if (g.k == 1) return constant(F_MAT1, 1, g.m);
            if (g.k == 2 && g.cbits.empty()) return constant(F_MAT2, 2, g.m);
            throw Unsupported("batch: dense gate form not supported");
        case Kind::Diag: {
            std::vector<cd> ph = g.m;
            ph.resize(4, cd(1, 0));
            return constant(F_DIAG, g.k, ph);
        }
        case Kind::Pair: {
            if (g.k == 4) return constant(F_PAIR4, 4, {g.m2[0], g.m2[1], g.m2[2], g.m2[3], g.gamma});
            if (g.k != 2) throw Unsupported("batch: pair gate width not supported");
            std::vector<cd> m(16, 0.0);
            for (int r = 0; r < 4; ++r) m[r * 4 + r] = g.gamma;
            m[g.pa * 4 + g.pa] = g.m2[0];
            m[g.pa * 4 + g.pb] = g.m2[1];
            m[g.pb * 4 + g.pa] = g.m2[2];
            m[g.pb * 4 + g.pb] = g.m2[3];
            return constant(F_MAT2, 2, m);
        }
        case Kind::Parity: {
            h.form = F_PARITY;
            h.nt = 0;
            h.gate = kConstGate;
            h.cmat = {g.pphase[0], g.pphase[1], 1.0, 1.0};
            return h;
        }
        default: throw Unsupported("batch: gate form not supported");
        }
    }
    // parameterised gate with a slot: coefficients synthesised on the device
    h.diff = true;
    h.gen = generator_of_gate(o.gate);
    switch (o.gate) {
    case B200SV_RX: case B200SV_RY: h.form = F_MAT1; h.nt = 1; break;
    case B200SV_RZ: h.form = F_DIAG; h.nt = 1; break;
    case B200SV_PhaseShift: h.form = F_DIAG; h.nt = 0; break;
    case B200SV_CRX: case B200SV_CRY: h.form = F_MAT1; h.nt = 1; break;
    case B200SV_CRZ: h.form = F_DIAG; h.nt = 1; break;
    case B200SV_ControlledPhaseShift: h.form = F_DIAG; h.nt = 0; break;
    case B200SV_IsingXX: case B200SV_IsingYY: case B200SV_IsingXY: case B200SV_SingleExcitation:
    case B200SV_SingleExcitationMinus: case B200SV_SingleExcitationPlus: h.form = F_MAT2; h.nt = 2; break;
    case B200SV_IsingZZ: h.form = F_DIAG; h.nt = 2; break;
    case B200SV_MultiRZ: h.form = F_PARITY; h.nt = 0; break;
    case B200SV_DoubleExcitation: case B200SV_DoubleExcitationMinus: case B200SV_DoubleExcitationPlus:
        h.form = F_PAIR4; h.nt = 4; break;
    default: throw Unsupported(std::string("batch: parameterised gate not supported: ") + gi.name);
    }
    return h;
}

struct Planned {
    std::vector<DCirc> circs;
    std::vector<DSeg> segs;
    std::vector<DOp> ops;
    std::vector<DTerm> terms;
    std::vector<double2> consts;
    std::vector<uint32_t> order;
    std::vector<double> gscale;
    std::vector<uint32_t> gslot_circ, gslot_col;
    std::vector<int64_t> gslot_param;
    size_t pool_a = 0, pool_b = 0;
    int max_kt = 1;
};

// coefficients in whole slots of 16 (a 4-wire matrix takes 16 consecutive slots)
uint32_t push_const(Planned &P, const std::vector<cd> &m) {
    const uint32_t idx = (uint32_t)(P.consts.size() / 16);
    const size_t n = std::max<size_t>(16, (m.size() + 15) / 16 * 16);
    for (size_t i = 0; i < n; ++i) {
        const cd z = i < m.size() ? m[i] : cd(0, 0);
        P.consts.push_back(make_double2(z.real(), z.imag()));
    }
    return idx;
}

// lower one host op into a device op with tile-local bit positions
DOp lower(Planned &P, const HostOp &h, const std::vector<int> &loc /* state bit -> tile bit */) {
    DOp d{};
    d.form = (uint8_t)h.form;
    d.gate = (uint8_t)(h.gate == kConstGate ? kConstGate : h.gate);
    d.inv = h.inv ? 1 : 0;
    d.nt = (uint8_t)h.nt;
    d.pslot = (int32_t)(h.gate == kConstGate ? -1 : h.pslot);
    d.gslot = -1;
    std::vector<uint32_t> lb(h.bits.size());
    for (size_t i = 0; i < h.bits.size(); ++i) lb[i] = (uint32_t)loc[h.bits[i]];
    uint32_t mb = 0;
    for (auto x : lb) mb = std::max(mb, x);
    d.maxbit = (uint8_t)mb;  // every form, swaps included: decides warp-local scheduling
    d.run = 1;
    // targets are the last nt bits of the reference wire order; the rest are controls
    const size_t nc = h.form == F_PARITY || h.form == F_NOOP ? 0 : lb.size() - h.nt;
    std::vector<uint32_t> tgt(lb.begin() + nc, lb.end()), ctl(lb.begin(), lb.begin() + nc);
    if (h.form == F_DIAG && h.nt == 0) {  // phase on all-ones of the listed bits
        ctl = lb;
        tgt.clear();
    }
    if (h.form == F_SWAP) {
        // X-type (nt == 1): swap rows 0/1 of the target; SWAP-type (nt == 2): rows 1/2
        std::vector<uint32_t> all = lb;
        std::sort(all.begin(), all.end());
        d.nb = (uint8_t)all.size();
        for (size_t j = 0; j < all.size(); ++j) d.low[j] = (uint16_t)((1u << all[j]) - 1);
        for (auto x : ctl) d.cmask |= 1u << x;
        if (h.nt == 1) {
            d.off[0] = 0;
            d.off[1] = 1u << tgt[0];
        } else {
            d.off[0] = 1u << tgt[1];  // row 01
            d.off[1] = 1u << tgt[0];  // row 10
        }
        d.cidx = 0;
        return d;
    }
    if (h.form == F_PARITY) {
        for (auto x : lb) d.pmask |= 1u << x;
        d.nb = 0;
    } else if (h.form == F_PAIR4 || h.form == F_MATK) {
        // every bit is a target; off[j] is target j's bit (matrix order)
        std::vector<uint32_t> all = lb;
        std::sort(all.begin(), all.end());
        d.nb = (uint8_t)all.size();
        for (size_t j = 0; j < all.size(); ++j) d.low[j] = (uint16_t)((1u << all[j]) - 1);
        for (size_t j = 0; j < lb.size(); ++j) d.off[j] = 1u << lb[j];
        d.nt = (uint8_t)lb.size();
    } else {
        std::vector<uint32_t> all = lb;
        std::sort(all.begin(), all.end());
        d.nb = (uint8_t)all.size();
        for (size_t j = 0; j < all.size(); ++j) d.low[j] = (uint16_t)((1u << all[j]) - 1);
        for (auto x : ctl) d.cmask |= 1u << x;
        const int nt = (int)tgt.size();
        for (int r = 0; r < (1 << nt); ++r) {
            uint32_t o = 0;
            for (int j = 0; j < nt; ++j)
                if (r & (1 << (nt - 1 - j))) o |= 1u << tgt[j];
            d.off[r] = o;
        }
        d.nt = (uint8_t)nt;
    }
    if (h.gate == kConstGate) d.cidx = push_const(P, h.cmat);
    if (h.diff && h.gen >= 0) {
        double sc = 0.0;
        // generator as a matrix on the gate's bits (all of them, controls included)
        // built with the plain-path compiler on a virtual register whose bits are the tile bits
        std::vector<uint32_t> vw(lb.size());
        const uint32_t vq = 32;
        for (size_t i = 0; i < lb.size(); ++i) vw[i] = vq - 1 - lb[i];
        GateDesc G = compile_generator((uint32_t)h.gen, vw.data(), (uint32_t)vw.size(), vq, &sc);
        d.gscale = -2.0 * sc * (h.inv ? -1.0 : 1.0);
        // single-wire generators get a code for the fused-run path
        switch (h.gen) {
        case 0: d.gcode = 4; break;  // PhaseShift: |1><1|
        case 1: d.gcode = 1; break;  // RX: X
        case 2: d.gcode = 2; break;  // RY: Y
        case 3: d.gcode = 3; break;  // RZ: Z
        default: d.gcode = 0; break;
        }
        if (G.kind == Kind::Parity) {
            d.gform = G_PARITY;
            d.pmask = (uint32_t)G.pmask;
        } else if (G.kind == Kind::Pair && G.k == 4) {
            // same bits and rows as the gate (F_PAIR4): Y on rows (0011, 1100), gamma elsewhere
            if (h.form != F_PAIR4 || G.tbits != lb || G.pa != 3 || G.pb != 12)
                throw Unsupported("batch: four-wire generator layout");
            d.gform = G_PAIR4;
            d.gk = G.gamma == cd(1, 0) ? 1 : G.gamma == cd(-1, 0) ? 2 : 0;
        } else {
            // expand to a dense matrix over G.tbits (k <= 2)
            const int k = G.k;
            if (k > 2) throw Unsupported("batch: generator wider than two wires");
            const int D = 1 << k;
            std::vector<cd> gm(D * D, 0.0);
            if (G.kind == Kind::Dense) gm = G.m;
            else if (G.kind == Kind::Diag) for (int r = 0; r < D; ++r) gm[r * D + r] = G.m[r];
            else if (G.kind == Kind::Pair) {
                for (int r = 0; r < D; ++r) gm[r * D + r] = G.gamma;
                gm[G.pa * D + G.pa] = G.m2[0];
                gm[G.pa * D + G.pb] = G.m2[1];
                gm[G.pb * D + G.pa] = G.m2[2];
                gm[G.pb * D + G.pb] = G.m2[3];
            }
            d.gform = G_MAT;
            d.gk = (uint8_t)k;
            std::vector<uint32_t> gb = G.tbits;
            std::vector<uint32_t> sorted = gb;
            std::sort(sorted.begin(), sorted.end());
            d.gnb = (uint8_t)sorted.size();
            for (size_t j = 0; j < sorted.size(); ++j) d.glow[j] = (uint16_t)((1u << sorted[j]) - 1);
            for (int r = 0; r < D; ++r) {
                uint32_t o = 0;
                for (int j = 0; j < k; ++j)
                    if (r & (1 << (k - 1 - j))) o |= 1u << gb[j];
                d.goff[r] = o;
            }
            d.gcidx = push_const(P, gm);
        }
    }
    return d;
}

// Single-wire gate whose generator (if any) acts on the same wire: it can join
// a run that is applied per amplitude pair in registers.
int run_bit(const DOp &d) {
    int bit = -1;
    if (d.form == F_MAT1 && d.nb == 1 && d.cmask == 0) bit = d.maxbit;
    else if (d.form == F_DIAG && d.nb == 1 && (d.nt == 1 ? d.cmask == 0 : d.nt == 0)) bit = d.maxbit;
    else if (d.form == F_SWAP && d.nt == 1 && d.nb == 1 && d.cmask == 0) bit = d.maxbit;
    if (bit < 0) return -1;
    if (d.gslot >= 0 && d.gcode == 0) return -1;
    return bit;
}

// Structure of a run member's matrix (the adjoint has the same structure).
uint8_t member_kind(const DOp &d, const double2 *consts) {
    if (d.form == F_SWAP) return MK_SWAP;
    if (d.form == F_DIAG) return d.nt == 1 ? MK_DIAG : MK_PHASE1;
    if (d.gate == B200SV_RY) return MK_REAL;
    if (d.gate == B200SV_RX) return MK_RX;
    if (d.gate == kConstGate) {  // classify a constant 2x2 by its entries
        const double2 *c = consts + (size_t)d.cidx * 16;
        auto zero = [](double2 z) { return z.x == 0.0 && z.y == 0.0; };
        if (zero(c[1]) && zero(c[2])) return MK_DIAG;
        bool real = true, rx = true;
        for (int i = 0; i < 4; ++i) real = real && c[i].y == 0.0;
        rx = c[0].y == 0.0 && c[3].y == 0.0 && c[1].x == 0.0 && c[2].x == 0.0;
        if (real) return MK_REAL;
        if (rx) return MK_RX;
    }
    return MK_GENERAL;
}

void mark_runs(DOp *ops, uint32_t n, const double2 *consts) {
    uint32_t i = 0;
    while (i < n) {
        const int b = run_bit(ops[i]);
        uint32_t j = i + 1;
        if (b >= 0)
            while (j < n && j - i < (uint32_t)kMaxRun && run_bit(ops[j]) == b) ++j;
        if (j - i >= 2) {
            ops[i].run = (uint8_t)(j - i);
            for (uint32_t q = i; q < j; ++q) {
                ops[q].rbit = (uint8_t)b;
                ops[q].mkind = member_kind(ops[q], consts);
            }
            for (uint32_t q = i + 1; q < j; ++q) {
                ops[q].run = 0;
                ops[q].back = (uint8_t)(q - i);
            }
        }
        i = j;
    }
}

// Pair adjacent runs of one segment for the forward sweep's exec_run2, greedily from the
// first run: equal length and pairing signature, different bits.
void mark_pairs(DOp *ops, uint32_t n) {
    struct RunRef {
        uint32_t head, len;
        int code;  // 0 when the signature does not pair
    };
    std::vector<RunRef> runs;
    for (uint32_t i = 0; i < n;) {
        if (ops[i].run < 2) {
            ++i;
            continue;
        }
        const uint32_t len = ops[i].run;
        int k[kMaxRun] = {0, 0, 0};
        bool general = false;
        for (uint32_t m = 0; m < len; ++m) {
            general = general || ops[i + m].mkind == MK_GENERAL;
            k[m] = ops[i + m].mkind;
        }
        RunRef rr{i, len, 0};
        const int sf = run_sig((int)len, k[0], 0, k[1], 0, k[2], 0);
        for (int code = 1; code <= 3 && !general; ++code)
            if (sf == pair_sig(code)) rr.code = code;
        ops[i].pair = 0;
        runs.push_back(rr);
        i += len;
    }
    for (size_t r = 0; r + 1 < runs.size();) {
        const RunRef &a = runs[r], &b = runs[r + 1];
        if (a.head + a.len == b.head && a.len == b.len && a.code != 0 && a.code == b.code &&
            ops[a.head].rbit != ops[b.head].rbit) {
            ops[a.head].pair = (uint8_t)a.code;
            r += 2;
        } else {
            ++r;
        }
    }
}

// Lowest state bits every tile keeps: 2^r contiguous amplitudes = 128 bytes.
uint64_t low_reserve_mask(int dtype, uint32_t kt) {
    const uint32_t r = std::min<uint32_t>(dtype == B200SV_C64 ? 4 : 3, kt > 4 ? kt - 4 : 0);
    return (uint64_t(1) << r) - 1;
}

Planned plan(const Batch &B, const Config &cfg, bool vjp) {
    Planned P;
    P.consts.reserve(1024);
    push_const(P, {});  // slot 0 unused
    const uint32_t nc = B.ncirc;
    std::vector<double> cost(nc);
    uint32_t out_begin = 0;
    for (uint32_t c = 0; c < nc; ++c) {
        const uint32_t n = B.nq[c];
        DCirc dc{};
        dc.n = n;
        const int live = vjp ? 2 : 1;
        (void)live;
        dc.kt = (uint32_t)std::min<int>(cfg.kt, (int)n);
        dc.resident = n <= (uint32_t)cfg.kt ? 1 : 0;
        dc.seg_begin = (uint32_t)P.segs.size();
        dc.nobs = B.nobs[c];
        dc.out_begin = out_begin;
        out_begin += B.nobs[c];
        dc.term_begin = (uint32_t)P.terms.size();
        for (auto t : B.hterms[c]) P.terms.push_back(t);
        dc.nterms = (uint32_t)B.hterms[c].size();
        // segmentation
        const auto &ops = B.hops[c];
        size_t i = 0;
        // tiles of a multi-tile circuit always hold the lowest state bits, so every
        // tile is made of contiguous runs of at least 128 bytes
        const uint64_t low = dc.resident ? 0 : low_reserve_mask(B.dtype, dc.kt);
        while (i < ops.size() || (i == 0 && ops.empty())) {
            uint64_t used = 0;
            size_t j = i;
            while (j < ops.size()) {
                uint64_t b = 0;
                for (auto x : ops[j].bits) b |= uint64_t(1) << x;
                if (popcount64(used | b) > (int)dc.kt || (popcount64(used | b | low) > (int)dc.kt && j > i)) break;
                if (j - i >= (size_t)kMaxSegOpsStaged) break;
                used |= b;
                ++j;
            }
            if (j == i && i < ops.size()) throw Unsupported("batch: gate wider than the tile");
            // local bits: used bits plus the lowest unused bits up to kt
            std::vector<uint32_t> L;
            for (uint32_t x = 0; x < n; ++x)
                if (used & (uint64_t(1) << x)) L.push_back(x);
            for (uint32_t x = 0; x < n && L.size() < dc.kt; ++x)
                if (!(used & (uint64_t(1) << x))) L.push_back(x);
            std::sort(L.begin(), L.end());
            DSeg s{};
            s.nl = (uint8_t)L.size();
            std::vector<int> loc(n, -1);
            for (size_t q = 0; q < L.size(); ++q) {
                s.lbits[q] = (uint8_t)L[q];
                loc[L[q]] = (int)q;
            }
            uint8_t ng = 0;
            for (uint32_t x = 0; x < n; ++x)
                if (loc[x] < 0) s.gbits[ng++] = (uint8_t)x;
            s.ng = ng;
            s.op_begin = (uint32_t)P.ops.size();
            s.nops = (uint32_t)(j - i);
            for (size_t q = i; q < j; ++q) {
                DOp d = lower(P, ops[q], loc);
                if (ops[q].diff && vjp) {
                    d.gslot = (int32_t)P.gscale.size();
                    P.gscale.push_back(d.gscale);
                    P.gslot_circ.push_back(c);
                    P.gslot_param.push_back(ops[q].pslot);
                }
                P.ops.push_back(d);
            }
            mark_runs(P.ops.data() + s.op_begin, s.nops, P.consts.data());
            mark_pairs(P.ops.data() + s.op_begin, s.nops);
            P.segs.push_back(s);
            if (ops.empty()) break;
            i = j;
        }
        dc.nseg = (uint32_t)(P.segs.size() - dc.seg_begin);
        if (!dc.resident) {
            dc.off_a = P.pool_a;
            P.pool_a += uint64_t(1) << n;
            if (vjp) {
                dc.off_b = P.pool_b;
                P.pool_b += uint64_t(1) << n;
            }
        }
        P.max_kt = std::max<int>(P.max_kt, (int)dc.kt);
        cost[c] = double(uint64_t(1) << n) * double(ops.size() + 1);
        P.circs.push_back(dc);
    }
    P.order.resize(nc);
    std::iota(P.order.begin(), P.order.end(), 0u);
    std::stable_sort(P.order.begin(), P.order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
    // per gslot column index within its circuit (param ops in op order)
    std::vector<uint32_t> col_count(nc, 0);
    P.gslot_col.resize(P.gslot_circ.size());
    for (size_t g = 0; g < P.gslot_circ.size(); ++g) P.gslot_col[g] = col_count[P.gslot_circ[g]]++;
    return P;
}

template <typename R> const void *batch_kernel_r(int mode, bool full) {
    if (full) return mode ? (const void *)k_batch<R, 1, true> : (const void *)k_batch<R, 0, true>;
    return mode ? (const void *)k_batch<R, 1, false> : (const void *)k_batch<R, 0, false>;
}
const void *batch_kernel(int dtype, int mode, bool full) {
    return dtype == B200SV_C64 ? batch_kernel_r<float>(mode, full) : batch_kernel_r<double>(mode, full);
}

template <typename T> void upload(Batch &B, T *&dst, const std::vector<T> &src) {
    dst = B.dalloc<T>(src.size());
    if (!src.empty())
        B200SV_CUDA(cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// Build the device program for a configuration (both forward and VJP share it:
// the VJP layout is a superset).
void build_program(Batch &B, const Config &cfg) {
    B.free_program();
    Planned P = plan(B, cfg, true);
    B.cfg = cfg;
    upload(B, B.d_circs, P.circs);
    upload(B, B.d_segs, P.segs);
    upload(B, B.d_ops, P.ops);
    upload(B, B.d_terms, P.terms);
    upload(B, B.d_consts, P.consts);
    upload(B, B.d_order, P.order);
    B.h_circs = P.circs;
    B.d_counter = B.dalloc<uint32_t>(1);
    B.pool_a_bytes = P.pool_a * B.amp();
    B.pool_b_bytes = P.pool_b * B.amp();
    B.d_pool_a = B.dalloc<unsigned char>(B.pool_a_bytes);
    B.d_pool_b = B.dalloc<unsigned char>(B.pool_b_bytes);
    B.ngslots = (uint32_t)P.gscale.size();
    const int nw = cfg.threads / 32;
    B.d_gradw = B.dalloc<double>((size_t)B.ngslots * nw);
    upload(B, B.d_gscale, P.gscale);
    // CSR param -> gslots
    std::vector<uint32_t> rowptr(B.nparams + 1, 0), cols;
    for (size_t g = 0; g < P.gslot_param.size(); ++g) {
        const int64_t p = P.gslot_param[g];
        if (p >= 0 && (uint64_t)p < B.nparams) rowptr[p + 1]++;
    }
    for (uint64_t p = 0; p < B.nparams; ++p) rowptr[p + 1] += rowptr[p];
    cols.resize(rowptr[B.nparams]);
    std::vector<uint32_t> fill(rowptr.begin(), rowptr.end() - 1);
    for (size_t g = 0; g < P.gslot_param.size(); ++g) {
        const int64_t p = P.gslot_param[g];
        if (p >= 0 && (uint64_t)p < B.nparams) cols[fill[p]++] = (uint32_t)g;
    }
    upload(B, B.d_rowptr, rowptr);
    upload(B, B.d_cols, cols);
    upload(B, B.d_gslot_circ, P.gslot_circ);
    upload(B, B.d_gslot_col, P.gslot_col);
    B.circ_ncols.assign(B.ncirc, 0);
    for (auto c : P.gslot_circ) B.circ_ncols[c]++;
    B.jac_base.assign(B.ncirc, 0);
    uint64_t acc = 0;
    for (uint32_t c = 0; c < B.ncirc; ++c) {
        B.jac_base[c] = acc;
        acc += (uint64_t)B.nobs[c] * B.circ_ncols[c];
    }
    B.jac_total = acc;
    upload(B, B.d_circ_ncols, B.circ_ncols);
    upload(B, B.d_jac_base, B.jac_base);
    B.d_dy_tmp = B.dalloc<double>(B.total_obs);
    B.d_params_in = B.dalloc<double>(B.nparams);
    B.d_params_fwd = B.dalloc<double>(B.nparams);
    B.d_cs = B.dalloc<double4>(B.nparams);
    B.nops_total = (uint32_t)P.ops.size();
    B.d_rcf = B.dalloc<unsigned char>(std::max<size_t>(1, P.ops.size()) * 4 * B.amp());
    B.d_fwd_valid = B.dalloc<int>(1);
    B.d_reuse = B.dalloc<int>(1);
    B200SV_CUDA(cudaMemset(B.d_fwd_valid, 0, sizeof(int)));
    B.d_dy_in = B.dalloc<double>(B.total_obs);
    B.d_out = B.dalloc<double>(B.total_obs);
    B.d_grad = B.dalloc<double>(B.nparams);
    B.smem_bytes = (size_t)2 * (size_t(1) << P.max_kt) * B.amp();
    int dev = 0, maxsm = 0, nsm = sm_count();
    B200SV_CUDA(cudaGetDevice(&dev));
    B200SV_CUDA(cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t static_smem = kObsPerPass * 32 * 8 + 2 * 16 * 16 + 64 + sizeof(DSeg) +
                               kMaxSegOpsStaged * (sizeof(DOp) + 4 * B.amp());
    if (B.smem_bytes + static_smem > (size_t)maxsm)
        throw Unsupported("batch: tile does not fit in shared memory; lower kt");
    B.full = false;
    for (const DOp &d : P.ops)
        if (d.form == F_MAT2 || d.form == F_PAIR4 || d.form == F_MATK || (d.gform == G_MAT && d.gk == 2) ||
            d.gform == G_PAIR4)
            B.full = true;
    int per_sm = 1 << 30;
    for (int mode = 0; mode < 2; ++mode) {
        const void *k = batch_kernel(B.dtype, mode, B.full);
        B200SV_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)B.smem_bytes));
        int m = 0;
        B200SV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k, cfg.threads, B.smem_bytes));
        per_sm = std::min(per_sm, m);
    }
    if (per_sm < 1) throw Unsupported("batch: launch configuration does not fit on an SM");
    B.grid = std::max(1, std::min<int>((int)B.ncirc, nsm * per_sm));
    B200SV_CUDA(cudaDeviceSynchronize());
}

// Per-parameter trigonometry for this launch (one k_trig pass over the batch parameters).
void launch_trig(Batch &B, const double *params, cudaStream_t st) {
    if (!B.nparams) return;
    const uint64_t nb = std::min<uint64_t>((B.nparams + 255) / 256, 4096);
    k_trig<<<(unsigned)nb, 256, 0, st>>>(params, B.nparams, B.d_cs);
    B200SV_CUDA(cudaGetLastError());
}

void launch_main(Batch &B, int mode, const double *dy, double *out, const int *reuse, cudaStream_t st) {
    KArgs A{};
    A.circs = B.d_circs;
    A.segs = B.d_segs;
    A.ops = B.d_ops;
    A.terms = B.d_terms;
    A.consts = B.d_consts;
    A.order = B.d_order;
    A.ncirc = B.ncirc;
    A.counter = B.d_counter;
    A.cs = B.d_cs;
    A.dy = dy;
    A.out = out;
    A.gradw = B.d_gradw;
    A.pool_a = B.d_pool_a;
    A.pool_b = B.d_pool_b;
    A.reuse = reuse;
    A.rcf = B.d_rcf;
    if (mode == 1 && B.nops_total) {
        const unsigned nb = std::max(1u, std::min(4096u, (B.nops_total + 255) / 256));
        if (B.dtype == B200SV_C64)
            k_rev_coeffs<float><<<nb, 256, 0, st>>>(B.d_ops, B.nops_total, B.d_cs, B.d_consts,
                                                     static_cast<C<float>(*)[4]>(B.d_rcf));
        else
            k_rev_coeffs<double><<<nb, 256, 0, st>>>(B.d_ops, B.nops_total, B.d_cs, B.d_consts,
                                                      static_cast<C<double>(*)[4]>(B.d_rcf));
        B200SV_CUDA(cudaGetLastError());
    }
    int mk = 1;
    for (auto &c : B.h_circs) mk = std::max<int>(mk, (int)c.kt);
    A.max_kt = mk;
    B200SV_CUDA(cudaMemsetAsync(B.d_counter, 0, sizeof(uint32_t), st));
    void *args[] = {&A};
    const void *k = batch_kernel(B.dtype, mode, B.full);
    B200SV_CUDA(cudaLaunchKernel(k, dim3(B.grid), dim3(B.cfg.threads), args, B.smem_bytes, st));
}

// Forward: expectation values; the final states of circuits wider than a tile stay
// in pool A, and a copy of the parameters marks them valid for the next VJP.
void enqueue_forward(Batch &B, cudaStream_t st) {
    launch_trig(B, B.d_params_in, st);
    launch_main(B, 0, nullptr, B.d_out, nullptr, st);
    if (B.nparams)
        B200SV_CUDA(cudaMemcpyAsync(B.d_params_fwd, B.d_params_in, B.nparams * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st));
    B200SV_CUDA(cudaMemsetAsync(B.d_fwd_valid, 1, sizeof(int), st));
}

// VJP: reuses pool A when it still holds the forward states of the same
// parameters (decided on the device, so the recorded graph stays valid), then
// invalidates it — the reverse sweep consumes those states.
void enqueue_vjp(Batch &B, cudaStream_t st) {
    launch_trig(B, B.d_params_in, st);
    B200SV_CUDA(cudaMemcpyAsync(B.d_reuse, B.d_fwd_valid, sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (B.nparams) {
        const uint64_t nb = std::min<uint64_t>((B.nparams + 255) / 256, 4096);
        k_params_equal<<<(unsigned)nb, 256, 0, st>>>(B.d_params_in, B.d_params_fwd, B.nparams, B.d_reuse);
        B200SV_CUDA(cudaGetLastError());
    }
    launch_main(B, 1, B.d_dy_in, nullptr, B.d_reuse, st);
    B200SV_CUDA(cudaMemsetAsync(B.d_fwd_valid, 0, sizeof(int), st));
    const int nw = B.cfg.threads / 32;
    const uint64_t np = std::max<uint64_t>(B.nparams, 1);
    k_grad_params<<<(unsigned)std::min<uint64_t>((np + 255) / 256, 4096), 256, 0, st>>>(
        B.d_rowptr, B.d_cols, B.d_gscale, B.d_gradw, nw, B.nparams, B.d_grad);
    B200SV_CUDA(cudaGetLastError());
}

template <class F> void run_maybe_graph(Batch &B, cudaGraphExec_t &exec, F &&enqueue) {
    cudaStream_t st = B.stream();
    if (!B.use_graphs) {
        enqueue(st);
        return;
    }
    if (!exec) {
        // Capture on the batch's private non-blocking stream (the legacy default
        // stream cannot be captured); the instantiated graph then launches on
        // the caller's stream, ordered with its other work.
        cudaGraph_t g = nullptr;
        B200SV_CUDA(cudaStreamBeginCapture(B.own, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue(B.own);
        } catch (...) {
            cudaStreamEndCapture(B.own, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        B200SV_CUDA(cudaStreamEndCapture(B.own, &g));
        const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        B200SV_CUDA(e);
    }
    B200SV_CUDA(cudaGraphLaunch(exec, st));
}

}  // namespace batch
}  // namespace b200sv

// =============================================================================
using namespace b200sv;
using namespace b200sv::batch;

struct b200sv_batch {
    std::unique_ptr<Batch> b;
};

extern "C" {

int b200sv_batch_create(int dtype, const b200sv_batch_circuit *circuits, uint32_t ncircuits, uint64_t nparams,
                        b200sv_batch_handle *out) {
    return run_guarded([&] {
        if (!out) throw ArgError("NULL output handle");
        if (dtype != B200SV_C64 && dtype != B200SV_C128) throw ArgError("dtype must be B200SV_C64 or B200SV_C128");
        if (ncircuits == 0 || !circuits) throw ArgError("a batch needs at least one circuit");
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            throw CudaError("no CUDA device is available (libb200sv has no CPU path)");
        }
        auto B = std::make_unique<Batch>();
        B->dtype = dtype;
        B->nparams = nparams;
        B->ncirc = ncircuits;
        B200SV_CUDA(cudaGetDevice(&B->device));
        B200SV_CUDA(cudaStreamCreateWithFlags(&B->own, cudaStreamNonBlocking));
        for (uint32_t c = 0; c < ncircuits; ++c) {
            const b200sv_batch_circuit &bc = circuits[c];
            if (bc.num_qubits < 1 || bc.num_qubits > 30) throw ArgError("batch circuits have 1..30 qubits");
            if (bc.nops && !bc.ops) throw ArgError("NULL ops");
            B->nq.push_back(bc.num_qubits);
            std::vector<HostOp> hv;
            for (uint32_t i = 0; i < bc.nops; ++i) {
                const int64_t ps = bc.param_index ? bc.param_index[i] : -1;
                if (ps >= 0 && (uint64_t)ps >= nparams) throw ArgError("batch: parameter index out of range");
                hv.push_back(make_hostop(bc.ops[i], ps, bc.num_qubits, dtype));
            }
            B->hops.push_back(std::move(hv));
            std::vector<DTerm> terms;
            uint32_t t_global = 0;
            for (uint32_t o = 0; o < bc.nobs; ++o) {
                for (uint32_t t = 0; t < bc.obs_nterms[o]; ++t, ++t_global) {
                    DTerm dt{};
                    dt.obs = o;
                    dt.coeff = bc.obs_coeffs[t_global];
                    uint64_t used = 0;
                    for (uint32_t q = bc.obs_offsets[t_global]; q < bc.obs_offsets[t_global + 1]; ++q) {
                        const uint32_t w = bc.obs_wires[q];
                        if (w >= bc.num_qubits) throw ArgError("batch: observable wire out of range");
                        const uint64_t bit = uint64_t(1) << bitpos(w, bc.num_qubits);
                        if (used & bit) throw ArgError("All wires in observables must be disjoint.");
                        used |= bit;
                        switch (bc.obs_paulis[q]) {
                        case 'I': break;
                        case 'X': dt.xmask |= bit; break;
                        case 'Y': dt.xmask |= bit; dt.zmask |= bit; dt.ny++; break;
                        case 'Z': dt.zmask |= bit; break;
                        default: throw ArgError("Pauli letters must be I, X, Y or Z");
                        }
                    }
                    terms.push_back(dt);
                }
            }
            B->hterms.push_back(std::move(terms));
            B->nobs.push_back(bc.nobs);
            B->total_obs += bc.nobs;
        }
        Config cfg;
        cfg.kt = dtype == B200SV_C64 ? 13 : 12;
        cfg.threads = 512;
        build_program(*B, cfg);
        auto *h = new b200sv_batch;
        h->b = std::move(B);
        *out = h;
    });
}

int b200sv_batch_destroy(b200sv_batch_handle b) {
    return run_guarded([&] {
        if (!b) return;
        cudaStreamSynchronize(b->b->stream());
        delete b;
    });
}

int b200sv_batch_set_stream(b200sv_batch_handle b, void *s) {
    return run_guarded([&] {
        if (!b) throw ArgError("NULL batch");
        // on a change of stream, the work issued on the previous one completes first
        if (!b->b->has_ext || b->b->ext != static_cast<cudaStream_t>(s))
            B200SV_CUDA(cudaStreamSynchronize(b->b->stream()));
        b->b->ext = static_cast<cudaStream_t>(s);
        b->b->has_ext = true;  // instantiated graphs launch on any stream
    });
}

int b200sv_batch_use_graphs(b200sv_batch_handle b, int enable) {
    return run_guarded([&] {
        if (!b) throw ArgError("NULL batch");
        b->b->use_graphs = enable != 0;
    });
}

int b200sv_batch_forward(b200sv_batch_handle bh, const double *params, double *out) {
    return run_guarded([&] {
        if (!bh) throw ArgError("NULL batch");
        Batch &B = *bh->b;
        if (B.nparams && !params) throw ArgError("NULL params");
        if (!out) throw ArgError("NULL output");
        cudaStream_t st = B.stream();
        if (B.nparams)
            B200SV_CUDA(cudaMemcpyAsync(B.d_params_in, params, B.nparams * sizeof(double), cudaMemcpyDeviceToDevice, st));
        run_maybe_graph(B, B.g_forward, [&](cudaStream_t s) { enqueue_forward(B, s); });
        B200SV_CUDA(cudaMemcpyAsync(out, B.d_out, B.total_obs * sizeof(double), cudaMemcpyDeviceToDevice, st));
        B.last_launches = 2;  // k_trig, k_batch
    });
}

int b200sv_batch_vjp(b200sv_batch_handle bh, const double *params, const double *dy, double *grad) {
    return run_guarded([&] {
        if (!bh) throw ArgError("NULL batch");
        Batch &B = *bh->b;
        if ((B.nparams && !params) || !dy || (B.nparams && !grad)) throw ArgError("NULL device buffer");
        cudaStream_t st = B.stream();
        if (B.nparams)
            B200SV_CUDA(cudaMemcpyAsync(B.d_params_in, params, B.nparams * sizeof(double), cudaMemcpyDeviceToDevice, st));
        B200SV_CUDA(cudaMemcpyAsync(B.d_dy_in, dy, B.total_obs * sizeof(double), cudaMemcpyDeviceToDevice, st));
        run_maybe_graph(B, B.g_vjp, [&](cudaStream_t s) { enqueue_vjp(B, s); });
        if (B.nparams)
            B200SV_CUDA(cudaMemcpyAsync(grad, B.d_grad, B.nparams * sizeof(double), cudaMemcpyDeviceToDevice, st));
        B.last_launches = 5;  // k_trig, k_params_equal, k_rev_coeffs, k_batch, k_grad_params
    });
}

int b200sv_batch_jacobian(b200sv_batch_handle bh, const double *params, double *jac) {
    return run_guarded([&] {
        if (!bh) throw ArgError("NULL batch");
        Batch &B = *bh->b;
        if ((B.nparams && !params) || !jac) throw ArgError("NULL device buffer");
        cudaStream_t st = B.stream();
        if (B.nparams)
            B200SV_CUDA(cudaMemcpyAsync(B.d_params_in, params, B.nparams * sizeof(double), cudaMemcpyDeviceToDevice, st));
        uint32_t maxobs = 0;
        for (auto n : B.nobs) maxobs = std::max(maxobs, n);
        const int nw = B.cfg.threads / 32;
        uint32_t launches = 1;
        B200SV_CUDA(cudaMemsetAsync(B.d_fwd_valid, 0, sizeof(int), st));
        launch_trig(B, B.d_params_in, st);
        for (uint32_t o = 0; o < maxobs; ++o) {
            k_onehot_dy<<<std::max(1u, (B.ncirc + 255) / 256), 256, 0, st>>>(B.d_dy_in, B.d_circs, B.ncirc, o);
            launch_main(B, 1, B.d_dy_in, nullptr, nullptr, st);
            if (B.ngslots)
                k_grad_scatter<<<std::max(1u, (B.ngslots + 255) / 256), 256, 0, st>>>(
                    B.d_gscale, B.d_gradw, nw, B.ngslots, o, B.d_gslot_circ, B.d_circs, B.d_jac_base,
                    B.d_gslot_col, B.d_circ_ncols, jac);
            B200SV_CUDA(cudaGetLastError());
            launches += 4;  // k_onehot_dy, k_rev_coeffs, k_batch, k_grad_scatter
        }
        B.last_launches = launches;
    });
}

int b200sv_batch_autotune(b200sv_batch_handle bh, const double *params, int *chosen) {
    return run_guarded([&] {
        if (!bh) throw ArgError("NULL batch");
        Batch &B = *bh->b;
        cudaStream_t st = B.stream();
        if (B.nparams)
            B200SV_CUDA(cudaMemcpyAsync(B.d_params_in, params, B.nparams * sizeof(double), cudaMemcpyDeviceToDevice, st));
        std::vector<Config> cands;
        const int kts_c64[] = {11, 12, 13};
        const int kts_c128[] = {10, 11, 12};
        for (int th : {256, 512})
            for (int i = 0; i < 3; ++i) cands.push_back(Config{th, B.dtype == B200SV_C64 ? kts_c64[i] : kts_c128[i]});
        float best = 1e30f;
        int best_i = -1;
        std::vector<double> saved_params(B.nparams);
        if (B.nparams)
            B200SV_CUDA(cudaMemcpy(saved_params.data(), B.d_params_in, B.nparams * sizeof(double), cudaMemcpyDeviceToHost));
        cudaEvent_t e0, e1;
        B200SV_CUDA(cudaEventCreate(&e0));
        B200SV_CUDA(cudaEventCreate(&e1));
        for (size_t i = 0; i < cands.size(); ++i) {
            try {
                build_program(B, cands[i]);
            } catch (const Unsupported &) {
                continue;
            }
            if (B.nparams)
                B200SV_CUDA(cudaMemcpy(B.d_params_in, saved_params.data(), B.nparams * sizeof(double), cudaMemcpyHostToDevice));
            B200SV_CUDA(cudaMemset(B.d_dy_in, 0, B.total_obs * sizeof(double)));
            // one training step as callers run it: forward values, then the VJP reusing the
            // forward's states; best of three after a warm-up step
            auto step = [&] {
                enqueue_forward(B, st);
                enqueue_vjp(B, st);
            };
            step();
            float ms = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                B200SV_CUDA(cudaEventRecord(e0, st));
                step();
                B200SV_CUDA(cudaEventRecord(e1, st));
                B200SV_CUDA(cudaEventSynchronize(e1));
                float t = 0;
                B200SV_CUDA(cudaEventElapsedTime(&t, e0, e1));
                ms = std::min(ms, t);
            }
            if (ms < best) {
                best = ms;
                best_i = (int)i;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (best_i < 0) throw Unsupported("batch autotune: no configuration fits");
        build_program(B, cands[best_i]);
        if (B.nparams)
            B200SV_CUDA(cudaMemcpy(B.d_params_in, saved_params.data(), B.nparams * sizeof(double), cudaMemcpyHostToDevice));
        if (chosen) *chosen = cands[best_i].threads * 100 + cands[best_i].kt;
    });
}

int b200sv_batch_last_launches(b200sv_batch_handle b, uint32_t *out) {
    return run_guarded([&] {
        if (!b || !out) throw ArgError("NULL argument");
        *out = b->b->last_launches;
    });
}

}  // extern "C"
