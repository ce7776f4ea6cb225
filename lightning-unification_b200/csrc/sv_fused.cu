// sv_fused.cu — one HBM pass for a run of gates on a single large state.
//
// The per-gate kernels (sv_gates.cu) read and write the whole state once per gate.
// Here gates whose wires fit in one shared-memory tile of 2^kt amplitudes form a
// segment: every CTA of a persistent grid takes tiles (the amplitudes that share the
// values of the n - kt bits outside the tile), applies all of the segment's gates to
// the tile and writes it back.  Tiles always contain the lowest state bits, so a tile is
// a set of contiguous 128-byte (or longer) runs, and tiles are double-buffered: cp.async
// brings the next tile in while the current one is computed and stored.
//
// Inside a tile the gates run in registers.  Each of the 512 threads holds A amplitudes
// (8 for complex128, 16 for complex64) that differ in a = log2(A) "register bits" of the
// tile; the other kt - a tile bits come from the thread index.  A phase is a run of gates
// whose target bits all lie in the phase's register bits: the threads load their
// amplitudes from shared memory once, apply every gate of the phase in registers and
// store them back once.  Diagonal gates (phases, controlled phases, MultiRZ) and control
// bits need no exchange at all, so they join any phase.  Only the hand-over between
// phases goes through shared memory, and the tile buffers are XOR-swizzled so that those
// exchanges are free of bank conflicts for most register-bit choices.
//
// Segments are formed with look-ahead: a gate joins the current segment when its bits fit
// the tile and it commutes with every earlier gate that was left out (disjoint bits, or
// both diagonal), so gates on wires that are already in the tile are pulled forward.
//
// Gate coefficients come from the same compiled GateDesc as the per-gate path (FP64 on
// the host, rounded once to the state's precision); complex64 outputs are compensated
// sums (CAcc<float>), as in the per-gate kernels.
#include <algorithm>
#include <cstring>
#include <functional>
#include <vector>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr int kFThreads = 512;
constexpr int kMaxGroupBits = 8;
constexpr int kMaxSegOps = 192;
constexpr int kMaxSegCoefs = 2048;

// Tile geometry: 2^kt amplitudes (64 KiB) per tile, A = 2^kt / 512 amplitudes per thread.
template <typename R> struct Geo;
template <> struct Geo<double> { static constexpr int kt = 12, a = 3, A = 8, reserve = 3; };
template <> struct Geo<float> { static constexpr int kt = 13, a = 4, A = 16, reserve = 4; };

// Shared-memory position of tile amplitude l.  complex128: the three low bits are XORed
// with bits 3..5, so eight threads whose amplitudes differ in any three of bits 0..5
// (bits s and s+3 not both) hit eight different 16-byte bank groups.  complex64: bits
// 1..3 XOR bits 4..6 (bit 0 stays, so the 16-byte pairs moved by cp.async stay together).
template <typename R> __host__ __device__ __forceinline__ uint32_t swz(uint32_t l);
template <> __host__ __device__ __forceinline__ uint32_t swz<double>(uint32_t l) { return l ^ ((l >> 3) & 7u); }
template <> __host__ __device__ __forceinline__ uint32_t swz<float>(uint32_t l) {
    return l ^ (((l >> 4) & 7u) << 1);
}

// ---- shared-memory forms (gates that do not fit the register bits) ---------------------

// One gate in tile-local bit positions.
struct alignas(16) FOp {
    int32_t kind;   // Kind
    int32_t k;      // target bits
    int32_t nb;     // group bits (targets and controls)
    int32_t coef;   // first coefficient (index into the segment's coefficients)
    uint32_t cmask; // controls, tile-local
    int32_t ra, rb; // Swap: exchanged rows; Pair: rows of the 2x2 block
    int32_t rest;   // Pair: multiply the other rows by gamma
    uint32_t low[kMaxGroupBits];  // (1 << pos) - 1 for the ascending group bit positions
    uint32_t off[16];             // row offsets: row r has bit (k-1-j) set for target j
    uint32_t pm_local;            // Parity: selected bits inside the tile (tile-local)
    uint32_t pad;
    uint64_t pm_global;           // Parity: selected bits outside the tile (state positions)
};

__device__ __forceinline__ uint32_t ins_group(uint32_t g, const uint32_t *low, int nb) {
#pragma unroll
    for (int j = 0; j < kMaxGroupBits; ++j) {
        if (j < nb) {
            const uint32_t lo = g & low[j];
            g = ((g ^ lo) << 1) | lo;
        }
    }
    return g;
}

struct OpRegs {
    uint32_t low[kMaxGroupBits];
    uint32_t off[16];
    uint32_t cmask;
    int nb;
};
template <int D> __device__ __forceinline__ OpRegs op_regs(const FOp &op) {
    OpRegs r;
#pragma unroll
    for (int j = 0; j < kMaxGroupBits; ++j) r.low[j] = op.low[j];
#pragma unroll
    for (int j = 0; j < 16; ++j) r.off[j] = j < D ? op.off[j] : 0u;
    r.cmask = op.cmask;
    r.nb = op.nb;
    return r;
}

// Givens block on two rows of a 2^k group, gamma on the other rows (double excitations):
// the only form that runs on the shared-memory tile instead of in registers.
template <typename R>
__device__ void f_pair(C<R> *s, const FOp &op, const C<R> *cf, int kt) {
    const OpRegs o = op_regs<16>(op);
    const int D = 1 << op.k, ra = op.ra, rb = op.rb, rest = op.rest;
    C<R> m[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) m[i] = cf[i];
    const uint32_t ng = 1u << (kt - o.nb);
    const uint32_t oa = op.off[ra], ob = op.off[rb];
    for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
        const uint32_t b = ins_group(g, o.low, o.nb) | o.cmask;
        const C<R> va = s[swz<R>(b + oa)], vb = s[swz<R>(b + ob)];
        CAcc<R> x, y;
        x.add(m[0], va);
        x.add(m[1], vb);
        y.add(m[2], va);
        y.add(m[3], vb);
        s[swz<R>(b + oa)] = x.get();
        s[swz<R>(b + ob)] = y.get();
        if (rest) {
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                if (r >= D || r == ra || r == rb) continue;
                CAcc<R> z;
                z.add(m[4], s[swz<R>(b + o.off[r])]);
                s[swz<R>(b + o.off[r])] = z.get();
            }
        }
    }
}

// ---- register forms --------------------------------------------------------------------

// A phase: the threads' register bits and the gates applied in registers.
struct alignas(16) RPhase {
    int32_t op_begin, nops;  // register ops (segment-local indices)
    int32_t fop;             // >= 0: the phase is one shared-memory op (segment-local FOp index)
    uint32_t comp;           // tile bits taken from the thread index (ascending); the rest are register bits
    uint32_t rdep[16];       // tile offset of register g (g's bits deposited into the register bits)
    uint32_t srdep[16];      // swz(rdep[g]): the swizzle is linear over XOR, so a register's shared-memory
                             // position is swz(thread part) ^ srdep[g]
    uint32_t ilow[4];        // (1 << register bit j) - 1, ascending: the thread part is the thread index
                             // with zeros inserted at the register bits
};

// the thread part of a phase's tile offsets: the thread index with a zero inserted at each of
// the phase's NA register bits (the thread index deposited into comp, in NA steps)
template <int NA> __device__ __forceinline__ uint32_t phase_base(uint32_t x, const RPhase &ph) {
#pragma unroll
    for (int j = 0; j < NA; ++j) {
        const uint32_t lo = x & ph.ilow[j];
        x = ((x ^ lo) << 1) | lo;
    }
    return x;
}

// Register op codes: form and, for the forms with targets, the register mask of the targets
// (index into the list of masks with that many bits).
enum RCode : int32_t {
    RC_DIAG = 0,     // phases indexed by up to three tile bits (controls folded into the table)
    RC_PARITY = 1,   // phase chosen by the parity of selected bits (MultiRZ)
    RC_DIAG_T = 2,   // RC_DIAG whose index bits are all thread bits: one factor for the thread
    RC_PARITY_T = 3, // RC_PARITY whose tile bits are all thread bits
    RC_DENSE1 = 16,  // + register bit
    RC_DENSE2 = 32,  // + index of the two-bit mask
    RC_DENSE3 = 48,  // + index of the three-bit mask
    RC_CTL = 128,    // added to a dense code: the gate has control bits
    RC_SWAP1 = 64,   // + register bit: exchange of rows 0 and 1, gated by controls
    RC_SWAP2 = 80,   // + index of the two-bit mask: exchange of |01> and |10>, gated by controls
    RC_PAIR2 = 96,   // + index of the two-bit mask: 2x2 block on |01>, |10>, gamma on |00>, |11>
};

struct alignas(16) ROp {
    int32_t code;
    int32_t coef;    // first coefficient (segment-local)
    uint32_t cmask;  // control bits (tile-local)
    int32_t kd;      // Diag: number of index bits (0..3); Pair: 1 when gamma != 1
    uint32_t p0, p1, p2; // Diag: tile positions of the index bits (p0 the most significant)
    uint32_t pm;     // Parity: tile-local bits
    uint64_t pmg;    // Parity: state bits outside the tile
    int32_t prod;    // adjoint sweep: generator product computed before this step (index), or -1
    int32_t pad3;
};

// masks of a-bit registers with two and three bits set, in increasing order
__host__ __device__ constexpr int mask2(int i) {
    return i == 0 ? 3 : i == 1 ? 5 : i == 2 ? 6 : i == 3 ? 9 : i == 4 ? 10 : 12;
}
__host__ __device__ constexpr int mask3(int i) { return i == 0 ? 7 : i == 1 ? 11 : i == 2 ? 13 : 14; }
// c's bits deposited into the set bits of mask (ascending)
__host__ __device__ constexpr int dep_c(int mask, int c) {
    int r = 0, j = 0;
    for (int b = 0; b < 8; ++b) {
        if ((mask >> b) & 1) {
            if ((c >> j) & 1) r |= 1 << b;
            ++j;
        }
    }
    return r;
}
__host__ __device__ constexpr int popc_c(int m) { return m == 0 ? 0 : (m & 1) + popc_c(m >> 1); }
__host__ __device__ constexpr int lowbit_c(int m) { return m & -m; }

// One complex product m * v, the value a one-term compensated sum (CAcc) returns: complex64
// forms each component with one FMA (cmul2), so the compensation word would stay zero.
template <typename R> __device__ __forceinline__ C<R> cprod(C<R> m, C<R> v) {
    if constexpr (sizeof(R) == 4) {
        return cmul2(m, v);
    } else {
        CAcc<R> acc;
        acc.add(m, v);
        return acc.get();
    }
}

template <typename R, int A, int MASK, bool CTL>
__device__ __forceinline__ void r_dense(C<R> (&v)[A], const uint32_t (&l)[A], uint32_t cmask,
                                        const C<R> *__restrict__ cf) {
    if constexpr (MASK < A) {
        constexpr int D = 1 << popc_c(MASK);
#pragma unroll
        for (int g = 0; g < A; ++g) {
            if (g & MASK) continue;
            if (CTL && (l[g] & cmask) != cmask) continue;
            C<R> x[D];
#pragma unroll
            for (int c = 0; c < D; ++c) x[c] = v[g | dep_c(MASK, c)];
#pragma unroll
            for (int r = 0; r < D; ++r) {
                CAcc<R> acc;
                acc.set(cf[r * D], x[0]);
#pragma unroll
                for (int c = 1; c < D; ++c) acc.add(cf[r * D + c], x[c]);
                v[g | dep_c(MASK, r)] = acc.get();
            }
        }
    }
}

template <typename R, int A, int MASK>
__device__ __forceinline__ void r_swap(C<R> (&v)[A], const uint32_t (&l)[A], uint32_t cmask) {
    if constexpr (MASK < A) {
        constexpr int LO = lowbit_c(MASK), HI = MASK ^ LO;  // one bit: rows 0, 1; two bits: |01>, |10>
#pragma unroll
        for (int g = 0; g < A; ++g) {
            if (g & MASK) continue;
            const bool on = (l[g] & cmask) == cmask;
            constexpr bool two = HI != 0;
            const int ia = two ? (g | LO) : g, ib = two ? (g | HI) : (g | LO);
            const C<R> x = v[ia], y = v[ib];
            v[ia] = on ? y : x;
            v[ib] = on ? x : y;
        }
    }
}

template <typename R, int A, int MASK>
__device__ __forceinline__ void r_pair(C<R> (&v)[A], const ROp &op, const C<R> *__restrict__ cf) {
    if constexpr (MASK < A) {
        constexpr int LO = lowbit_c(MASK), HI = MASK ^ LO;
        const C<R> m0 = cf[0], m1 = cf[1], m2 = cf[2], m3 = cf[3], gm = cf[4];
        const bool rest = op.kd != 0;
#pragma unroll
        for (int g = 0; g < A; ++g) {
            if (g & MASK) continue;
            const C<R> va = v[g | LO], vb = v[g | HI];
            CAcc<R> x, y;
            x.set(m0, va);
            x.add(m1, vb);
            y.set(m2, va);
            y.add(m3, vb);
            v[g | LO] = x.get();
            v[g | HI] = y.get();
            if (rest) {
                v[g] = cprod<R>(gm, v[g]);
                v[g | MASK] = cprod<R>(gm, v[g | MASK]);
            }
        }
    }
}

// phases indexed by up to three tile bits; bits beyond kd read a position-31 bit (always 0)
template <typename R, int A>
__device__ __forceinline__ void r_diag(C<R> (&v)[A], const uint32_t (&l)[A], const ROp &op,
                                       const C<R> *__restrict__ cf) {
    const uint32_t p0 = op.p0, p1 = op.p1, p2 = op.p2;
#pragma unroll
    for (int g = 0; g < A; ++g) {
        const uint32_t x = l[g];
        const uint32_t idx = (((x >> p0) & 1u) << 2) | (((x >> p1) & 1u) << 1) | ((x >> p2) & 1u);
        v[g] = cprod<R>(cf[idx], v[g]);
    }
}

template <typename R, int A>
__device__ __forceinline__ void r_parity(C<R> (&v)[A], const uint32_t (&l)[A], const ROp &op,
                                         const C<R> *__restrict__ cf, uint64_t tbase) {
    const int tp = __popcll(tbase & op.pmg) & 1;
    const C<R> ph0 = cf[tp], ph1 = cf[tp ^ 1];
#pragma unroll
    for (int g = 0; g < A; ++g) v[g] = cprod<R>((__popc(l[g] & op.pm) & 1) ? ph1 : ph0, v[g]);
}

// A diagonal step whose index bits all come from the thread index multiplies every amplitude
// the thread holds by the same factor.  Such a scalar commutes with every step of the phase
// (they act linearly within the thread's registers), so the factors are multiplied into one
// value tf, applied once when the phase ends: one product per step and thread instead of one
// per amplitude, with as many roundings per amplitude as applying the steps one by one.
template <typename R, int A>
__device__ __forceinline__ void run_rop(C<R> (&v)[A], const uint32_t (&l)[A], const ROp &op,
                                        const C<R> *__restrict__ scf, uint64_t tbase, uint32_t base, C<R> &tf,
                                        bool &has_tf) {
    const C<R> *cf = scf + op.coef;
    switch (op.code) {
    case RC_DIAG_T: {
        const uint32_t idx = (((base >> op.p0) & 1u) << 2) | (((base >> op.p1) & 1u) << 1) | ((base >> op.p2) & 1u);
        tf = has_tf ? cprod<R>(cf[idx], tf) : cf[idx];
        has_tf = true;
        break;
    }
    case RC_PARITY_T: {
        const int par = (__popcll(tbase & op.pmg) + __popc(base & op.pm)) & 1;
        tf = has_tf ? cprod<R>(cf[par], tf) : cf[par];
        has_tf = true;
        break;
    }
    case RC_DIAG: r_diag<R, A>(v, l, op, cf); break;
    case RC_PARITY: r_parity<R, A>(v, l, op, cf, tbase); break;
    case RC_DENSE1 + 0: r_dense<R, A, 1, false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE1 + 0: r_dense<R, A, 1, true>(v, l, op.cmask, cf); break;
    case RC_DENSE1 + 1: r_dense<R, A, 2, false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE1 + 1: r_dense<R, A, 2, true>(v, l, op.cmask, cf); break;
    case RC_DENSE1 + 2: r_dense<R, A, 4, false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE1 + 2: r_dense<R, A, 4, true>(v, l, op.cmask, cf); break;
    case RC_DENSE1 + 3: r_dense<R, A, 8, false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE1 + 3: r_dense<R, A, 8, true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 0: r_dense<R, A, mask2(0), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 0: r_dense<R, A, mask2(0), true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 1: r_dense<R, A, mask2(1), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 1: r_dense<R, A, mask2(1), true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 2: r_dense<R, A, mask2(2), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 2: r_dense<R, A, mask2(2), true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 3: r_dense<R, A, mask2(3), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 3: r_dense<R, A, mask2(3), true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 4: r_dense<R, A, mask2(4), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 4: r_dense<R, A, mask2(4), true>(v, l, op.cmask, cf); break;
    case RC_DENSE2 + 5: r_dense<R, A, mask2(5), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE2 + 5: r_dense<R, A, mask2(5), true>(v, l, op.cmask, cf); break;
    case RC_DENSE3 + 0: r_dense<R, A, mask3(0), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE3 + 0: r_dense<R, A, mask3(0), true>(v, l, op.cmask, cf); break;
    case RC_DENSE3 + 1: r_dense<R, A, mask3(1), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE3 + 1: r_dense<R, A, mask3(1), true>(v, l, op.cmask, cf); break;
    case RC_DENSE3 + 2: r_dense<R, A, mask3(2), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE3 + 2: r_dense<R, A, mask3(2), true>(v, l, op.cmask, cf); break;
    case RC_DENSE3 + 3: r_dense<R, A, mask3(3), false>(v, l, op.cmask, cf); break;
    case RC_CTL + RC_DENSE3 + 3: r_dense<R, A, mask3(3), true>(v, l, op.cmask, cf); break;
    case RC_SWAP1 + 0: r_swap<R, A, 1>(v, l, op.cmask); break;
    case RC_SWAP1 + 1: r_swap<R, A, 2>(v, l, op.cmask); break;
    case RC_SWAP1 + 2: r_swap<R, A, 4>(v, l, op.cmask); break;
    case RC_SWAP1 + 3: r_swap<R, A, 8>(v, l, op.cmask); break;
    case RC_SWAP2 + 0: r_swap<R, A, mask2(0)>(v, l, op.cmask); break;
    case RC_SWAP2 + 1: r_swap<R, A, mask2(1)>(v, l, op.cmask); break;
    case RC_SWAP2 + 2: r_swap<R, A, mask2(2)>(v, l, op.cmask); break;
    case RC_SWAP2 + 3: r_swap<R, A, mask2(3)>(v, l, op.cmask); break;
    case RC_SWAP2 + 4: r_swap<R, A, mask2(4)>(v, l, op.cmask); break;
    case RC_SWAP2 + 5: r_swap<R, A, mask2(5)>(v, l, op.cmask); break;
    case RC_PAIR2 + 0: r_pair<R, A, mask2(0)>(v, op, cf); break;
    case RC_PAIR2 + 1: r_pair<R, A, mask2(1)>(v, op, cf); break;
    case RC_PAIR2 + 2: r_pair<R, A, mask2(2)>(v, op, cf); break;
    case RC_PAIR2 + 3: r_pair<R, A, mask2(3)>(v, op, cf); break;
    case RC_PAIR2 + 4: r_pair<R, A, mask2(4)>(v, op, cf); break;
    case RC_PAIR2 + 5: r_pair<R, A, mask2(5)>(v, op, cf); break;
    default: break;
    }
}

__device__ __forceinline__ uint64_t deposit(uint64_t x, const uint8_t *pos, int nbits) {
    uint64_t r = 0;
    for (int i = 0; i < nbits; ++i) r |= ((x >> i) & 1u) << pos[i];
    return r;
}


struct SegArgs {
    const RPhase *phases;
    const ROp *rops;
    const FOp *fops;
    const void *coefs;
    int nph, nrop, nfop, ncoef;
    int ng;
    uint8_t lbits[16];  // state position of tile bit i (ascending)
    uint8_t gbits[48];  // state positions of the bits outside the tile (ascending)
};

template <typename T> __device__ __forceinline__ void stage(T *dst, const T *src, int n) {
    static_assert(sizeof(T) % 4 == 0, "staged records are whole words");
    const uint32_t *s = reinterpret_cast<const uint32_t *>(src);
    uint32_t *d = reinterpret_cast<uint32_t *>(dst);
    const int words = n * (int)(sizeof(T) / 4);
    for (int i = threadIdx.x; i < words; i += blockDim.x) d[i] = s[i];
}

// One segment over all tiles.  Shared memory: two swizzled tile buffers, then the segment's
// phases, register ops, shared-memory ops and coefficients.  A tile is moved in 16-byte
// chunks (V amplitudes each, V = 16 / the amplitude size); chunk c of a thread is
// c = threadIdx.x + j * blockDim.x, j < A / V.
template <typename R>
__global__ void __launch_bounds__(kFThreads, 1) k_fused(C<R> *__restrict__ state, SegArgs a, uint64_t ntiles) {
    constexpr int KT = Geo<R>::kt, A = Geo<R>::A;
    constexpr uint32_t TN = 1u << KT;
    constexpr int V = 16 / (int)sizeof(C<R>);
    constexpr int PER = (int)(TN / V) / kFThreads;  // 16-byte chunks per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint8_t s_lbits[16], s_gbits[48];
    __shared__ uint64_t s_hi[PER];  // state offset of chunk row j (the same for every thread)
    C<R> *const buf0 = reinterpret_cast<C<R> *>(smem_raw);
    RPhase *sph = reinterpret_cast<RPhase *>(smem_raw + 2 * sizeof(C<R>) * TN);
    ROp *srop = reinterpret_cast<ROp *>(sph + a.nph);
    FOp *sfop = reinterpret_cast<FOp *>(srop + a.nrop);
    C<R> *scf = reinterpret_cast<C<R> *>(sfop + a.nfop);
    if (threadIdx.x == 0) {  // constant indices keep the parameter arrays out of local memory
#pragma unroll
        for (int i = 0; i < 16; ++i) s_lbits[i] = a.lbits[i];
#pragma unroll
        for (int i = 0; i < 48; ++i) s_gbits[i] = a.gbits[i];
    }
    stage(sph, a.phases, a.nph);
    stage(srop, a.rops, a.nrop);
    stage(sfop, a.fops, a.nfop);
    stage(scf, static_cast<const C<R> *>(a.coefs), a.ncoef);
    __syncthreads();
    // address parts of the tile moves: chunk c = threadIdx.x + j * 512 -> tile amplitude c * V
    if (threadIdx.x < PER) s_hi[threadIdx.x] = deposit((uint64_t)threadIdx.x * kFThreads * V, s_lbits, KT);
    __syncthreads();
    const uint64_t lo = deposit((uint64_t)threadIdx.x * V, s_lbits, KT);
    // swizzled shared-memory position of chunk j of this thread
    auto sw = [&](int j) { return swz<R>((threadIdx.x + (uint32_t)j * kFThreads) * V); };

    uint64_t t = blockIdx.x;
    uint32_t cur = 0;
    uint64_t tb_cur = 0;  // state offset of tile t (deposited once, when the tile is prefetched)
    if (t < ntiles) {
        tb_cur = deposit(t, s_gbits, a.ng);
#pragma unroll
        for (int j = 0; j < PER; ++j) cp_async16(buf0 + sw(j), state + (tb_cur | lo | s_hi[j]));
    }
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        const uint64_t tnext = t + gridDim.x;
        uint64_t tb_next = 0;
        if (tnext < ntiles) {
            tb_next = deposit(tnext, s_gbits, a.ng);
            C<R> *dst = buf0 + (cur ^ 1u) * TN;
#pragma unroll
            for (int j = 0; j < PER; ++j) cp_async16(dst + sw(j), state + (tb_next | lo | s_hi[j]));
        }
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        C<R> *s = buf0 + cur * TN;
        const uint64_t tbase = tb_cur;
        for (int p = 0; p < a.nph; ++p) {
            const RPhase &ph = sph[p];
            if (ph.fop >= 0) {
                const FOp &f = sfop[ph.fop];
                f_pair<R>(s, f, scf + f.coef, KT);
                __syncthreads();
                continue;
            }
            const uint32_t base = phase_base<Geo<R>::a>(threadIdx.x, ph);
            const uint32_t sbase = swz<R>(base);
            uint32_t l[A];
            C<R> v[A];
#pragma unroll
            for (int g = 0; g < A; ++g) l[g] = base | ph.rdep[g];
#pragma unroll
            for (int g = 0; g < A; ++g) v[g] = s[sbase ^ ph.srdep[g]];
            const int oe = ph.op_begin + ph.nops;
            C<R> tf = mk<R>(1, 0);
            bool has_tf = false;
            for (int o = ph.op_begin; o < oe; ++o) run_rop<R, A>(v, l, srop[o], scf, tbase, base, tf, has_tf);
            if (has_tf) {
#pragma unroll
                for (int g = 0; g < A; ++g) v[g] = cprod<R>(tf, v[g]);
            }
#pragma unroll
            for (int g = 0; g < A; ++g) s[sbase ^ ph.srdep[g]] = v[g];
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const float4 x = *reinterpret_cast<const float4 *>(s + sw(j));
            *reinterpret_cast<float4 *>(state + (tbase | lo | s_hi[j])) = x;
        }
        __syncthreads();  // the buffer is refilled next iteration
        cur ^= 1u;
        tb_cur = tb_next;
    }
    cp_async_wait0();
}

template <typename R> C<R> to_r(const cd &z) { return mk<R>((R)z.real(), (R)z.imag()); }

// Bits a descriptor touches (targets, controls, parity bits): gates with disjoint bit sets commute.
uint64_t dep_bits(const GateDesc &g) {
    uint64_t b = g.pmask;
    for (auto x : g.tbits) b |= uint64_t(1) << x;
    for (auto x : g.cbits) b |= uint64_t(1) << x;
    return b;
}
bool is_diagonal(const GateDesc &g) { return g.kind == Kind::Diag || g.kind == Kind::Parity || g.kind == Kind::Noop; }

// Tile bits (targets and controls) of a descriptor the tile kernel covers; false when the
// descriptor has to run on its own (wide dense matrices and the like).
bool tile_bits(const GateDesc &g, uint64_t &bits) {
    bits = 0;
    switch (g.kind) {
    case Kind::Noop: return true;
    case Kind::Parity: return true;
    case Kind::Dense: if (g.k < 1 || g.k > 3) return false; break;
    case Kind::Diag: if (g.k > 2) return false; break;
    case Kind::Swap: if (g.k < 1 || g.k > 2) return false; break;
    case Kind::Pair: if (g.k != 1 && g.k != 2 && g.k != 4) return false; break;
    default: return false;
    }
    if ((int)(g.tbits.size() + g.cbits.size()) > kMaxGroupBits) return false;
    for (auto b : g.tbits) bits |= uint64_t(1) << b;
    for (auto b : g.cbits) bits |= uint64_t(1) << b;
    return true;
}

int coef_count(const GateDesc &g) {
    switch (g.kind) {
    case Kind::Dense: return 1 << (2 * g.k);
    case Kind::Diag: return 8;  // a table over up to three bits (targets and controls)
    case Kind::Pair: return 5;
    case Kind::Parity: return 2;
    default: return 0;
    }
}

// ---- composing consecutive gates ---------------------------------------------------------
// Consecutive gates on one bit (RZ RY RZ of a Rot, H then RX, ...) are multiplied on the host
// in FP64 into one 2x2 step, and consecutive diagonal gates on at most two bits into one
// diagonal step; both need fewer operations than the gates one by one.  Wider products
// would trade cheap register steps for denser matrices, so they are not formed.

bool fusable(const GateDesc &g) {
    uint64_t b;
    return (g.kind == Kind::Dense || g.kind == Kind::Diag || g.kind == Kind::Swap || g.kind == Kind::Pair) &&
           tile_bits(g, b) && __builtin_popcountll(b) <= 3;
}

// apply g to a vector over the state bits pb (small index bit k-1-j <-> state bit pb[j])
void apply_small(const GateDesc &g, const std::vector<uint32_t> &pb, std::vector<cd> &v) {
    const int k = (int)pb.size();
    auto small = [&](uint32_t sb) {
        for (int j = 0; j < k; ++j)
            if (pb[j] == sb) return 1u << (k - 1 - j);
        return 0u;
    };
    uint32_t cm = 0, tall = 0;
    for (auto c : g.cbits) cm |= small(c);
    const int kg = (int)g.tbits.size();
    std::vector<uint32_t> tm(kg);
    for (int j = 0; j < kg; ++j) tall |= (tm[j] = small(g.tbits[j]));
    auto off = [&](uint32_t r) {
        uint32_t o = 0;
        for (int j = 0; j < kg; ++j)
            if ((r >> (kg - 1 - j)) & 1u) o |= tm[j];
        return o;
    };
    const uint32_t D = 1u << kg;
    for (uint32_t base = 0; base < (1u << k); ++base) {
        if ((base & cm) != cm || (base & tall) != 0) continue;
        switch (g.kind) {
        case Kind::Dense: {
            std::vector<cd> u(D), w(D, cd(0, 0));
            for (uint32_t r = 0; r < D; ++r) u[r] = v[base | off(r)];
            for (uint32_t r = 0; r < D; ++r)
                for (uint32_t c = 0; c < D; ++c) w[r] += g.m[r * D + c] * u[c];
            for (uint32_t r = 0; r < D; ++r) v[base | off(r)] = w[r];
            break;
        }
        case Kind::Diag:
            for (uint32_t r = 0; r < D; ++r) v[base | off(r)] *= g.m[r];
            break;
        case Kind::Swap:
            std::swap(v[base | off(g.sa)], v[base | off(g.sb)]);
            break;
        case Kind::Pair: {
            const cd a = v[base | off(g.pa)], b = v[base | off(g.pb)];
            v[base | off(g.pa)] = g.m2[0] * a + g.m2[1] * b;
            v[base | off(g.pb)] = g.m2[2] * a + g.m2[3] * b;
            for (uint32_t r = 0; r < D; ++r)
                if (r != g.pa && r != g.pb) v[base | off(r)] *= g.gamma;
            break;
        }
        default: break;
        }
    }
}

GateDesc compose(const std::vector<const GateDesc *> &gs, uint64_t bits) {
    GateDesc out;
    for (int b = 63; b >= 0; --b)
        if ((bits >> b) & 1) out.tbits.push_back((uint32_t)b);
    const int k = (int)out.tbits.size();
    const uint32_t D = 1u << k;
    std::vector<cd> M(D * D);
    for (uint32_t col = 0; col < D; ++col) {
        std::vector<cd> e(D, cd(0, 0));
        e[col] = cd(1, 0);
        for (const GateDesc *g : gs) apply_small(*g, out.tbits, e);
        for (uint32_t row = 0; row < D; ++row) M[row * D + col] = e[row];
    }
    bool diagonal = k <= 2;
    for (uint32_t r = 0; r < D && diagonal; ++r)
        for (uint32_t c = 0; c < D; ++c)
            if (r != c && M[r * D + c] != cd(0, 0)) diagonal = false;
    out.k = k;
    if (diagonal) {
        out.kind = Kind::Diag;
        for (uint32_t r = 0; r < D; ++r) out.m.push_back(M[r * D + r]);
    } else {
        out.kind = Kind::Dense;
        out.m = M;
    }
    return out;
}

std::vector<GateDesc> compose_runs(const std::vector<const GateDesc *> &in) {
    std::vector<GateDesc> out;
    size_t a = 0;
    while (a < in.size()) {
        uint64_t bits = 0, b1 = 0;
        if (!fusable(*in[a])) {
            out.push_back(*in[a++]);
            continue;
        }
        tile_bits(*in[a], bits);
        bool alldiag = in[a]->kind == Kind::Diag;
        size_t b = a + 1;
        while (b < in.size() && fusable(*in[b]) && tile_bits(*in[b], b1)) {
            const uint64_t nb = bits | b1;
            const bool nd = alldiag && in[b]->kind == Kind::Diag;
            if (!(__builtin_popcountll(nb) <= 1 || (nd && __builtin_popcountll(nb) <= 2))) break;
            bits = nb;
            alldiag = nd;
            ++b;
        }
        if (b - a == 1) out.push_back(*in[a]);
        else out.push_back(compose(std::vector<const GateDesc *>(in.begin() + a, in.begin() + b), bits));
        a = b;
    }
    return out;
}

// ---- lowering a segment into phases ------------------------------------------------------

template <typename R> struct SegCode {
    std::vector<RPhase> phases;
    std::vector<ROp> rops;
    std::vector<FOp> fops;
    std::vector<C<R>> coefs;
};

template <typename R>
FOp lower_fop(const GateDesc &g, const std::vector<int> &loc, std::vector<C<R>> &coefs) {
    FOp f{};
    f.kind = (int)g.kind;
    f.k = g.k;
    f.coef = (int32_t)coefs.size();
    std::vector<uint32_t> grp;
    for (auto b : g.tbits) grp.push_back((uint32_t)loc[b]);
    for (auto b : g.cbits) {
        grp.push_back((uint32_t)loc[b]);
        f.cmask |= 1u << loc[b];
    }
    std::sort(grp.begin(), grp.end());
    f.nb = (int)grp.size();
    for (size_t j = 0; j < grp.size(); ++j) f.low[j] = (1u << grp[j]) - 1;
    const int k = (int)g.tbits.size();
    for (int r = 0; r < (1 << k); ++r) {
        uint32_t o = 0;
        for (int j = 0; j < k; ++j)
            if (r & (1 << (k - 1 - j))) o |= 1u << loc[g.tbits[j]];
        f.off[r] = o;
    }
    f.ra = (int)g.pa;
    f.rb = (int)g.pb;
    for (auto &z : g.m2) coefs.push_back(to_r<R>(z));
    coefs.push_back(to_r<R>(g.gamma));
    f.rest = g.gamma != cd(1.0, 0.0) ? 1 : 0;
    return f;
}

// register targets a descriptor needs in its phase (tile-local mask), or -1 for the
// shared-memory form, 0 for the forms that work on any register bits
template <typename R> int64_t reg_targets(const GateDesc &g, const std::vector<int> &loc) {
    if (g.kind == Kind::Diag || g.kind == Kind::Parity || g.kind == Kind::Noop) return 0;
    if (g.kind == Kind::Pair && g.k == 4) return -1;
    uint64_t m = 0;
    for (auto b : g.tbits) m |= uint64_t(1) << loc[b];
    return (int64_t)m;
}

// hook(i, rop, rpos) runs before op i's record is stored (rpos: tile bit -> register bit)
using RopHook = std::function<void(size_t, ROp &, const int *)>;

template <typename R, typename G = Geo<R>>
void lower_phase(SegCode<R> &sc, uint32_t rmask, const std::vector<const GateDesc *> &ops,
                 const std::vector<int> &loc, const RopHook &hook = nullptr) {
    constexpr int KT = G::kt, a = G::a, A = G::A;
    // pad the register bits to a bits with the highest free tile bits
    for (int b = KT - 1; b >= 0 && __builtin_popcount(rmask) < a; --b)
        if (!((rmask >> b) & 1)) rmask |= 1u << b;
    int rpos[32];  // tile bit -> register bit
    int rb[8];
    {
        int j = 0;
        for (int b = 0; b < KT; ++b) {
            rpos[b] = -1;
            if ((rmask >> b) & 1) {
                rpos[b] = j;
                rb[j++] = b;
            }
        }
    }
    RPhase ph{};
    ph.op_begin = (int32_t)sc.rops.size();
    ph.fop = -1;
    ph.comp = ((1u << KT) - 1) & ~rmask;
    for (int j = 0; j < a; ++j) ph.ilow[j] = (1u << rb[j]) - 1;
    for (int g = 0; g < A; ++g) {
        uint32_t o = 0;
        for (int j = 0; j < a; ++j)
            if ((g >> j) & 1) o |= 1u << rb[j];
        ph.rdep[g] = o;
        ph.srdep[g] = swz<R>(o);
    }
    auto index_of = [](int m, int bits) {
        for (int i = 0; i < 6; ++i)
            if ((bits == 2 ? mask2(i) : mask3(i)) == m) return i;
        return -1;
    };
    auto emit = [&](size_t i, ROp &r) {
        if (hook) hook(i, r, rpos);
        sc.rops.push_back(r);
    };
    for (size_t oi = 0; oi < ops.size(); ++oi) {
        const GateDesc &g = *ops[oi];
        if (g.kind == Kind::Noop) continue;
        ROp r{};
        r.prod = -1;
        r.coef = (int32_t)sc.coefs.size();
        for (auto b : g.cbits) r.cmask |= 1u << loc[b];
        if (g.kind == Kind::Diag) {
            // one table over the target bits then the control bits: entry 1 where a control is clear
            r.code = RC_DIAG;
            r.cmask = 0;
            std::vector<uint32_t> ib(g.tbits.begin(), g.tbits.end());
            ib.insert(ib.end(), g.cbits.begin(), g.cbits.end());
            if (ib.size() > 3) throw Unsupported("fused diagonal step over more than three bits");
            r.kd = (int32_t)ib.size();
            uint32_t pos[3] = {31, 31, 31};
            for (size_t j = 0; j < ib.size(); ++j) pos[j] = (uint32_t)loc[ib[j]];
            r.p0 = pos[0];
            r.p1 = pos[1];
            r.p2 = pos[2];
            uint32_t used = 0;
            for (size_t j = 0; j < ib.size(); ++j) used |= 1u << pos[j];
            if ((used & rmask) == 0) r.code = RC_DIAG_T;  // thread bits only (also with no index bits)
            const int kt_ = g.k, kc = (int)g.cbits.size();
            for (int idx = 0; idx < 8; ++idx) {
                // idx bit (2 - j) holds index bit j; absent bits are zero in every address
                int t = 0;
                bool all_c = true;
                for (int j = 0; j < kt_ + kc; ++j) {
                    const int bit = (idx >> (2 - j)) & 1;
                    if (j < kt_) t = (t << 1) | bit;
                    else if (!bit) all_c = false;
                }
                sc.coefs.push_back(to_r<R>(all_c ? g.m[t] : cd(1.0, 0.0)));
            }
            emit(oi, r);
            continue;
        }
        if (g.kind == Kind::Parity) {
            r.code = RC_PARITY;
            for (int b = 0; b < 64; ++b) {
                if (!((g.pmask >> b) & 1)) continue;
                if (loc[b] >= 0) r.pm |= 1u << loc[b];
                else r.pmg |= uint64_t(1) << b;
            }
            if ((r.pm & rmask) == 0) r.code = RC_PARITY_T;
            sc.coefs.push_back(to_r<R>(g.pphase[0]));
            sc.coefs.push_back(to_r<R>(g.pphase[1]));
            emit(oi, r);
            continue;
        }
        // register bit of each target, and the target mask over the register bits
        const int k = (int)g.tbits.size();
        std::vector<int> regb(k);
        int mask = 0;
        for (int j = 0; j < k; ++j) {
            regb[j] = rpos[loc[g.tbits[j]]];
            mask |= 1 << regb[j];
        }
        if (g.kind == Kind::Swap) {
            r.code = k == 1 ? RC_SWAP1 + regb[0] : RC_SWAP2 + index_of(mask, 2);
            emit(oi, r);
            continue;
        }
        if (g.kind == Kind::Pair && k == 2) {
            // rows pa = 1 (tbits[0] clear, tbits[1] set) and pb = 2; canonical rows: the lower
            // register bit first
            r.code = RC_PAIR2 + index_of(mask, 2);
            r.kd = g.gamma != cd(1.0, 0.0) ? 1 : 0;
            const bool pa_low = regb[1] < regb[0];
            const cd m00 = g.m2[0], m01 = g.m2[1], m10 = g.m2[2], m11 = g.m2[3];
            const cd blk[4] = {pa_low ? m00 : m11, pa_low ? m01 : m10, pa_low ? m10 : m01, pa_low ? m11 : m00};
            for (auto &z : blk) sc.coefs.push_back(to_r<R>(z));
            sc.coefs.push_back(to_r<R>(g.gamma));
            emit(oi, r);
            continue;
        }
        // Dense (and the one-bit Pair form): canonical matrix, index bit i <-> i-th lowest mask bit
        std::vector<cd> m;
        if (g.kind == Kind::Pair) m = {g.m2[0], g.m2[1], g.m2[2], g.m2[3]};
        else m = g.m;
        const int D = 1 << k;
        std::vector<int> rank(k);  // position of regb[j] among the mask's set bits
        for (int j = 0; j < k; ++j) rank[j] = __builtin_popcount(mask & ((1 << regb[j]) - 1));
        auto orig = [&](int c) {
            int o = 0;
            for (int j = 0; j < k; ++j)
                if ((c >> rank[j]) & 1) o |= 1 << (k - 1 - j);
            return o;
        };
        for (int rr = 0; rr < D; ++rr)
            for (int cc = 0; cc < D; ++cc) sc.coefs.push_back(to_r<R>(m[orig(rr) * D + orig(cc)]));
        r.code = k == 1 ? RC_DENSE1 + regb[0] : k == 2 ? RC_DENSE2 + index_of(mask, 2) : RC_DENSE3 + index_of(mask, 3);
        if (r.cmask) r.code += RC_CTL;
        emit(oi, r);
    }
    ph.nops = (int32_t)sc.rops.size() - ph.op_begin;
    sc.phases.push_back(ph);
}

// Phases of one segment.  Gates commute when their bit sets are disjoint or both are
// diagonal, so a phase takes every gate that is ready (no earlier gate left behind shares a
// bit with it, unless both are diagonal) and whose targets still fit the register bits,
// scanning the segment in order until nothing more fits; the next phase starts from the
// earliest gate left.  A gate of the shared-memory form runs as a phase of its own once it
// is ready and no register gate can move.
template <typename R>
void lower_segment(SegCode<R> &sc, const std::vector<GateDesc> &ops, const std::vector<int> &loc) {
    constexpr int a = Geo<R>::a;
    const size_t n = ops.size();
    std::vector<int64_t> tgt(n);
    std::vector<uint64_t> bits(n);
    std::vector<char> diag(n), done(n, 0);
    for (size_t i = 0; i < n; ++i) {
        tgt[i] = reg_targets<R>(ops[i], loc);
        bits[i] = dep_bits(ops[i]);
        diag[i] = is_diagonal(ops[i]);
        if (ops[i].kind == Kind::Noop) done[i] = 1;
    }
    auto ready = [&](size_t i) {
        for (size_t j = 0; j < i; ++j)
            if (!done[j] && (bits[j] & bits[i]) && !(diag[j] && diag[i])) return false;
        return true;
    };
    size_t left = 0;
    for (size_t i = 0; i < n; ++i) left += done[i] ? 0 : 1;
    while (left > 0) {
        std::vector<const GateDesc *> cur;
        uint32_t rmask = 0;
        for (bool progress = true; progress;) {
            progress = false;
            for (size_t i = 0; i < n; ++i) {
                if (done[i] || tgt[i] < 0 || !ready(i)) continue;
                const uint32_t need = (uint32_t)tgt[i];
                if (__builtin_popcount(rmask | need) > a) continue;
                rmask |= need;
                cur.push_back(&ops[i]);
                done[i] = 1;
                --left;
                progress = true;
            }
        }
        if (!cur.empty()) {
            lower_phase<R>(sc, rmask, cur, loc);
            continue;
        }
        // no register gate can move: the earliest ready shared-memory gate goes next
        size_t i = 0;
        while (i < n && (done[i] || tgt[i] >= 0 || !ready(i))) ++i;
        if (i == n) throw Unsupported("fused phase planning made no progress");
        RPhase ph{};
        ph.fop = (int32_t)sc.fops.size();
        sc.fops.push_back(lower_fop<R>(ops[i], loc, sc.coefs));
        sc.phases.push_back(ph);
        done[i] = 1;
        --left;
    }
}

struct Segment {
    std::vector<uint8_t> lbits, gbits;
    uint32_t ph_begin = 0, nph = 0, rop_begin = 0, nrop = 0, fop_begin = 0, nfop = 0, coef_begin = 0, ncoef = 0;
};

template <typename R>
void run_fused(void *state, uint32_t nq, const std::vector<GateDesc> &descs,
               const std::function<void(const GateDesc &)> &apply_single, cudaStream_t st) {
    constexpr int kt = Geo<R>::kt;
    if ((int)nq < kt) throw Unsupported("state narrower than the fused tile");
    const uint64_t low = (uint64_t(1) << Geo<R>::reserve) - 1;  // 128 contiguous bytes in every tile
    struct Piece {
        bool seg;
        Segment s;
        size_t desc;
    };
    std::vector<Piece> pieces;
    SegCode<R> sc;
    const size_t nd = descs.size();
    std::vector<char> done(nd, 0);
    size_t first = 0;
    while (true) {
        while (first < nd && (done[first] || descs[first].kind == Kind::Noop)) ++first;
        if (first >= nd) break;
        uint64_t b = 0;
        if (!tile_bits(descs[first], b)) {
            pieces.push_back(Piece{false, {}, first});
            done[first] = 1;
            continue;
        }
        // look-ahead: take every later gate that fits and commutes with the gates left out
        uint64_t used = 0, blocked_any = 0, blocked_nondiag = 0;
        int nops = 0, ncf = 0;
        std::vector<size_t> take;
        for (size_t j = first; j < nd; ++j) {
            if (done[j] || descs[j].kind == Kind::Noop) continue;
            const GateDesc &g = descs[j];
            const uint64_t db = dep_bits(g);
            const bool diagonal = is_diagonal(g);
            const bool blocked = (db & blocked_nondiag) || (!diagonal && (db & blocked_any));
            bool fits = false;
            if (!blocked && tile_bits(g, b) && __builtin_popcountll(used | b | low) <= kt &&
                nops + 1 <= kMaxSegOps && ncf + coef_count(g) <= kMaxSegCoefs)
                fits = true;
            if (fits) {
                used |= b;
                ++nops;
                ncf += coef_count(g);
                take.push_back(j);
            } else {
                blocked_any |= db;
                if (!diagonal) blocked_nondiag |= db;
                if (__builtin_popcountll(blocked_any) >= (int)nq && blocked_nondiag == blocked_any) break;
            }
        }
        Segment sg;
        std::vector<int> loc(nq, -1);
        uint64_t inl = used | low;
        for (uint32_t x = 0; x < nq && __builtin_popcountll(inl) < kt; ++x) inl |= uint64_t(1) << x;
        for (uint32_t x = 0; x < nq; ++x) {
            if ((inl >> x) & 1) {
                loc[x] = (int)sg.lbits.size();
                sg.lbits.push_back((uint8_t)x);
            } else {
                sg.gbits.push_back((uint8_t)x);
            }
        }
        std::vector<const GateDesc *> seg;
        for (size_t j : take) {
            seg.push_back(&descs[j]);
            done[j] = 1;
        }
        const std::vector<GateDesc> fused = compose_runs(seg);
        sg.ph_begin = (uint32_t)sc.phases.size();
        sg.rop_begin = (uint32_t)sc.rops.size();
        sg.fop_begin = (uint32_t)sc.fops.size();
        sg.coef_begin = (uint32_t)sc.coefs.size();
        SegCode<R> local;
        lower_segment<R>(local, fused, loc);
        sc.phases.insert(sc.phases.end(), local.phases.begin(), local.phases.end());
        sc.rops.insert(sc.rops.end(), local.rops.begin(), local.rops.end());
        sc.fops.insert(sc.fops.end(), local.fops.begin(), local.fops.end());
        sc.coefs.insert(sc.coefs.end(), local.coefs.begin(), local.coefs.end());
        sg.nph = (uint32_t)local.phases.size();
        sg.nrop = (uint32_t)local.rops.size();
        sg.nfop = (uint32_t)local.fops.size();
        sg.ncoef = (uint32_t)local.coefs.size();
        pieces.push_back(Piece{true, sg, 0});
    }
    if (sc.phases.empty()) {
        for (auto &p : pieces) apply_single(descs[p.desc]);
        return;
    }
    // one device copy of every segment's records
    const size_t bph = sc.phases.size() * sizeof(RPhase), brop = sc.rops.size() * sizeof(ROp),
                 bfop = sc.fops.size() * sizeof(FOp), bcf = sc.coefs.size() * sizeof(C<R>);
    std::vector<unsigned char> blob(bph + brop + bfop + bcf + 16);
    std::memcpy(blob.data(), sc.phases.data(), bph);
    if (brop) std::memcpy(blob.data() + bph, sc.rops.data(), brop);
    if (bfop) std::memcpy(blob.data() + bph + brop, sc.fops.data(), bfop);
    if (bcf) std::memcpy(blob.data() + bph + brop + bfop, sc.coefs.data(), bcf);
    unsigned char *d_blob = nullptr;
    B200SV_CUDA(cudaMallocAsync((void **)&d_blob, blob.size(), st));
    struct Free {
        void *p;
        cudaStream_t s;
        ~Free() { cudaFreeAsync(p, s); }
    } fr{d_blob, st};
    B200SV_CUDA(cudaMemcpyAsync(d_blob, blob.data(), blob.size(), cudaMemcpyHostToDevice, st));
    const RPhase *d_ph = reinterpret_cast<const RPhase *>(d_blob);
    const ROp *d_rop = reinterpret_cast<const ROp *>(d_blob + bph);
    const FOp *d_fop = reinterpret_cast<const FOp *>(d_blob + bph + brop);
    const C<R> *d_cf = reinterpret_cast<const C<R> *>(d_blob + bph + brop + bfop);
    const size_t tile_bytes = sizeof(C<R>) << kt;
    auto seg_smem = [&](const Segment &s) {
        return 2 * tile_bytes + s.nph * sizeof(RPhase) + s.nrop * sizeof(ROp) + s.nfop * sizeof(FOp) +
               s.ncoef * sizeof(C<R>);
    };
    size_t smem_max = 0;
    for (const Piece &p : pieces)
        if (p.seg) smem_max = std::max(smem_max, seg_smem(p.s));
    // at most 192 ops per segment: 128 KiB of tiles + 192 x (160 + 48) B + 32 KiB of coefficients
    // (+ 160 B per double excitation)
    if (smem_max > 227 * 1024) throw Unsupported("fused segment records exceed shared memory");
    B200SV_CUDA(cudaFuncSetAttribute(k_fused<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    const uint64_t ntiles = uint64_t(1) << (nq - kt);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sm_count());
    for (const Piece &p : pieces) {
        if (!p.seg) {
            apply_single(descs[p.desc]);
            continue;
        }
        SegArgs a{};
        a.phases = d_ph + p.s.ph_begin;
        a.rops = d_rop + p.s.rop_begin;
        a.fops = d_fop + p.s.fop_begin;
        a.coefs = d_cf + p.s.coef_begin;
        a.nph = (int)p.s.nph;
        a.nrop = (int)p.s.nrop;
        a.nfop = (int)p.s.nfop;
        a.ncoef = (int)p.s.ncoef;
        a.ng = (int)p.s.gbits.size();
        std::memcpy(a.lbits, p.s.lbits.data(), p.s.lbits.size());
        std::memcpy(a.gbits, p.s.gbits.data(), p.s.gbits.size());
        k_fused<R><<<grid, kFThreads, seg_smem(p.s), st>>>(static_cast<C<R> *>(state), a, ntiles);
        B200SV_CUDA(cudaGetLastError());
    }
}

// ==== fused adjoint sweep ====================================================================
// The reverse sweep of the adjoint method (AdjointJacobianLQubit.hpp:212-335) over lambda
// and one bra: for each op, from the last, the product -2 scale Im<bra|G|lambda> when the op
// is differentiated, then the op's inverse on both states.  Runs of these steps whose bits
// fit a tile run as one pass over both states: the tile holds 2^kt amplitudes of each state,
// each thread A of each in registers (fewer than the forward kernel: two states share the
// register budget), and the phases apply each step to both states.  A product is formed per
// thread in FP64, summed over the warp with shuffles and added to the warp's slot of the
// step's accumulator in shared memory; after its tiles each CTA writes the sum of its warps'
// slots (fixed order), and a finalize kernel adds the CTAs' values (fixed order), so results
// are reproducible run to run.

template <typename R> struct GeoA;
template <> struct GeoA<double> { static constexpr int kt = 11, a = 2, A = 4, reserve = 3; };
template <> struct GeoA<float> { static constexpr int kt = 12, a = 3, A = 8, reserve = 4; };

constexpr int kMaxAdjItems = 96;
constexpr int kMaxAdjCoefs = 1024;
constexpr int kWarps = kFThreads / 32;

enum PCode : int32_t { PG_DIAG = 0, PG_PARITY = 1, PG_PAIR1 = 16 /* + register bit */ };

struct alignas(16) PProd {
    int32_t kind;
    int32_t item;   // accumulator row (differentiated step of the segment)
    int32_t coef;   // first FP64 coefficient (segment-local)
    uint32_t p0, p1, p2, pm;
    uint32_t pad;
    uint64_t pmg;
};

struct AdjSegArgs {
    const RPhase *phases;
    const ROp *rops;
    const PProd *prods;
    const void *coefs;      // gate coefficients (C<R>)
    const double2 *gcoefs;  // generator coefficients (FP64)
    int nph, nrop, nprod, ncoef, ngcoef, nitems;
    int ng;
    uint8_t lbits[16];
    uint8_t gbits[48];
};

__device__ __forceinline__ double im_conj(double2 w, double2 v) { return w.x * v.y - w.y * v.x; }
__device__ __forceinline__ double re_conj(double2 w, double2 v) { return w.x * v.x + w.y * v.y; }

// sum over this thread's amplitude groups of Im(conj(w) . G v), FP64
template <typename R, int A, int BIT>
__device__ __forceinline__ double prod_pair1(const C<R> (&v)[A], const C<R> (&w)[A], const double2 *__restrict__ m) {
    double p = 0.0;
    if constexpr ((1 << BIT) < A) {
        constexpr int B = 1 << BIT;
#pragma unroll
        for (int g = 0; g < A; ++g) {
            if (g & B) continue;
            const double2 v0 = widen<R>(v[g]), v1 = widen<R>(v[g | B]);
            const double2 w0 = widen<R>(w[g]), w1 = widen<R>(w[g | B]);
            // (G v)_r = m[2r] v0 + m[2r+1] v1
            const double2 g0 = make_double2(m[0].x * v0.x - m[0].y * v0.y + m[1].x * v1.x - m[1].y * v1.y,
                                            m[0].x * v0.y + m[0].y * v0.x + m[1].x * v1.y + m[1].y * v1.x);
            const double2 g1 = make_double2(m[2].x * v0.x - m[2].y * v0.y + m[3].x * v1.x - m[3].y * v1.y,
                                            m[2].x * v0.y + m[2].y * v0.x + m[3].x * v1.y + m[3].y * v1.x);
            p += im_conj(w0, g0) + im_conj(w1, g1);
        }
    }
    return p;
}

template <typename R, int A>
__device__ __forceinline__ double r_product(const C<R> (&v)[A], const C<R> (&w)[A], const uint32_t (&l)[A],
                                            const PProd &q, const double2 *__restrict__ gcf, uint64_t tbase) {
    const double2 *m = gcf + q.coef;
    double p = 0.0;
    switch (q.kind) {
    case PG_DIAG:
#pragma unroll
        for (int g = 0; g < A; ++g) {
            const uint32_t x = l[g];
            const uint32_t idx = (((x >> q.p0) & 1u) << 2) | (((x >> q.p1) & 1u) << 1) | ((x >> q.p2) & 1u);
            const double2 d = m[idx], vv = widen<R>(v[g]), ww = widen<R>(w[g]);
            p += d.x * im_conj(ww, vv) + d.y * re_conj(ww, vv);
        }
        break;
    case PG_PARITY: {
        const int tp = __popcll(tbase & q.pmg) & 1;
#pragma unroll
        for (int g = 0; g < A; ++g) {
            const double2 d = m[(__popc(l[g] & q.pm) & 1) ^ tp], vv = widen<R>(v[g]), ww = widen<R>(w[g]);
            p += d.x * im_conj(ww, vv) + d.y * re_conj(ww, vv);
        }
        break;
    }
    case PG_PAIR1 + 0: p = prod_pair1<R, A, 0>(v, w, m); break;
    case PG_PAIR1 + 1: p = prod_pair1<R, A, 1>(v, w, m); break;
    case PG_PAIR1 + 2: p = prod_pair1<R, A, 2>(v, w, m); break;
    default: break;
    }
    return p;
}

template <typename R>
__global__ void __launch_bounds__(kFThreads, 1) k_fused_adj(C<R> *__restrict__ lam, C<R> *__restrict__ bra,
                                                            AdjSegArgs a, uint64_t ntiles, double *partials) {
    constexpr int KT = GeoA<R>::kt, A = GeoA<R>::A;
    constexpr uint32_t TN = 1u << KT;
    constexpr int V = 16 / (int)sizeof(C<R>);
    constexpr int PER = (int)(TN / V) / kFThreads;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint8_t s_lbits[16], s_gbits[48];
    __shared__ uint64_t s_hi[PER];
    // buffers: [cur][state] tiles of TN amplitudes
    C<R> *const buf = reinterpret_cast<C<R> *>(smem_raw);
    RPhase *sph = reinterpret_cast<RPhase *>(smem_raw + 4 * sizeof(C<R>) * TN);
    ROp *srop = reinterpret_cast<ROp *>(sph + a.nph);
    PProd *sprod = reinterpret_cast<PProd *>(srop + a.nrop);
    double2 *sgcf = reinterpret_cast<double2 *>(sprod + a.nprod);
    double *sacc = reinterpret_cast<double *>(sgcf + a.ngcoef);
    C<R> *scf = reinterpret_cast<C<R> *>(sacc + (size_t)a.nitems * kWarps);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 16; ++i) s_lbits[i] = a.lbits[i];
#pragma unroll
        for (int i = 0; i < 48; ++i) s_gbits[i] = a.gbits[i];
    }
    stage(sph, a.phases, a.nph);
    stage(srop, a.rops, a.nrop);
    stage(sprod, a.prods, a.nprod);
    stage(sgcf, a.gcoefs, a.ngcoef);
    stage(scf, static_cast<const C<R> *>(a.coefs), a.ncoef);
    for (int i = threadIdx.x; i < a.nitems * kWarps; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    if (threadIdx.x < PER) s_hi[threadIdx.x] = deposit((uint64_t)threadIdx.x * kFThreads * V, s_lbits, KT);
    __syncthreads();
    const uint64_t lo = deposit((uint64_t)threadIdx.x * V, s_lbits, KT);
    auto sw = [&](int j) { return swz<R>((threadIdx.x + (uint32_t)j * kFThreads) * V); };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    uint64_t t = blockIdx.x;
    uint32_t cur = 0;
    auto load = [&](uint64_t tile, uint32_t b) {
        const uint64_t tb = deposit(tile, s_gbits, a.ng);
        C<R> *dl = buf + (2 * b) * TN, *db = buf + (2 * b + 1) * TN;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            cp_async16(dl + sw(j), lam + (tb | lo | s_hi[j]));
            cp_async16(db + sw(j), bra + (tb | lo | s_hi[j]));
        }
    };
    if (t < ntiles) load(t, 0);
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        const uint64_t tnext = t + gridDim.x;
        if (tnext < ntiles) load(tnext, cur ^ 1u);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        C<R> *sl = buf + (2 * cur) * TN, *sb = buf + (2 * cur + 1) * TN;
        const uint64_t tbase = deposit(t, s_gbits, a.ng);
        for (int p = 0; p < a.nph; ++p) {
            const RPhase &ph = sph[p];
            const uint32_t base = phase_base<GeoA<R>::a>(threadIdx.x, ph);
            const uint32_t sbase = swz<R>(base);
            uint32_t l[A];
            C<R> v[A], w[A];
#pragma unroll
            for (int g = 0; g < A; ++g) l[g] = base | ph.rdep[g];
#pragma unroll
            for (int g = 0; g < A; ++g) {
                v[g] = sl[sbase ^ ph.srdep[g]];
                w[g] = sb[sbase ^ ph.srdep[g]];
            }
            C<R> tf = mk<R>(1, 0), tf2 = mk<R>(1, 0);
            bool has_tf = false, unused = false;
            const int oe = ph.op_begin + ph.nops;
            for (int o = ph.op_begin; o < oe; ++o) {
                const ROp &op = srop[o];
                if (op.prod >= 0) {
                    // the deferred thread factor is a unit scalar common to both states: the
                    // product does not see it
                    const PProd &q = sprod[op.prod];
                    double pr = r_product<R, A>(v, w, l, q, sgcf, tbase);
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) pr += __shfl_xor_sync(0xffffffffu, pr, off);
                    if (lane == 0) sacc[q.item * kWarps + warp] += pr;
                }
                run_rop<R, A>(v, l, op, scf, tbase, base, tf, has_tf);
                if (op.code != RC_DIAG_T && op.code != RC_PARITY_T)
                    run_rop<R, A>(w, l, op, scf, tbase, base, tf2, unused);
            }
            if (has_tf) {
#pragma unroll
                for (int g = 0; g < A; ++g) {
                    v[g] = cprod<R>(tf, v[g]);
                    w[g] = cprod<R>(tf, w[g]);
                }
            }
#pragma unroll
            for (int g = 0; g < A; ++g) {
                sl[sbase ^ ph.srdep[g]] = v[g];
                sb[sbase ^ ph.srdep[g]] = w[g];
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            *reinterpret_cast<float4 *>(lam + (tbase | lo | s_hi[j])) = *reinterpret_cast<const float4 *>(sl + sw(j));
            *reinterpret_cast<float4 *>(bra + (tbase | lo | s_hi[j])) = *reinterpret_cast<const float4 *>(sb + sw(j));
        }
        __syncthreads();
        cur ^= 1u;
    }
    cp_async_wait0();
    __syncthreads();
    for (int i = threadIdx.x; i < a.nitems; i += blockDim.x) {
        double sum = 0.0;
        for (int wv = 0; wv < kWarps; ++wv) sum += sacc[i * kWarps + wv];
        partials[(size_t)i * gridDim.x + blockIdx.x] = sum;
    }
}

// jac[col[i]] = alpha[i] * sum_b partials[i * nb + b]   (one block per item, fixed order)
__global__ void k_adj_fused_final(const double *__restrict__ partials, int nb, const double *__restrict__ alpha,
                                  const int64_t *__restrict__ col, double *__restrict__ jac) {
    __shared__ double sm[32];
    double s[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s[0] += partials[(size_t)blockIdx.x * nb + b];
    block_reduce<1>(s, sm);
    if (threadIdx.x == 0) jac[col[blockIdx.x]] = alpha[blockIdx.x] * s[0];
}

// generator -> product record (false when the product has no register form)
bool lower_prod(const GateDesc &G, const std::vector<int> &loc, const int *rpos, int item, PProd &q,
                std::vector<double2> &gcf) {
    q = PProd{};
    q.item = item;
    q.coef = (int32_t)gcf.size();
    auto d2 = [](const cd &z) { return make_double2(z.real(), z.imag()); };
    switch (G.kind) {
    case Kind::Diag: {
        if (!G.cbits.empty() || G.k > 3) return false;
        uint32_t pos[3] = {31, 31, 31};
        for (int j = 0; j < G.k; ++j) pos[j] = (uint32_t)loc[G.tbits[j]];
        q.kind = PG_DIAG;
        q.p0 = pos[0];
        q.p1 = pos[1];
        q.p2 = pos[2];
        for (int idx = 0; idx < 8; ++idx) {
            int t = 0;
            for (int j = 0; j < G.k; ++j) t = (t << 1) | ((idx >> (2 - j)) & 1);
            gcf.push_back(d2(G.m[t]));
        }
        return true;
    }
    case Kind::Parity:
        q.kind = PG_PARITY;
        for (int b = 0; b < 64; ++b) {
            if (!((G.pmask >> b) & 1)) continue;
            if (b < (int)loc.size() && loc[b] >= 0) q.pm |= 1u << loc[b];
            else q.pmg |= uint64_t(1) << b;
        }
        gcf.push_back(d2(G.pphase[0]));
        gcf.push_back(d2(G.pphase[1]));
        return true;
    case Kind::Pair:
        if (G.k != 1 || !rpos) return false;
        q.kind = PG_PAIR1 + rpos[loc[G.tbits[0]]];
        for (int i = 0; i < 4; ++i) gcf.push_back(d2(G.m2[i]));
        return true;
    default: return false;
    }
}

// the product of an adjoint item has a register form: which register bit it needs (0: none), or -1
int64_t prod_targets(const GateDesc &G, const std::vector<int> &loc) {
    switch (G.kind) {
    case Kind::Diag: return G.cbits.empty() && G.k <= 3 ? 0 : -1;
    case Kind::Parity: return 0;
    case Kind::Pair: return G.k == 1 ? (int64_t)(uint64_t(1) << loc[G.tbits[0]]) : -1;
    default: return -1;
    }
}

template <typename R>
void run_fused_adjoint(void *lam, void *bra, uint32_t nq, const std::vector<AdjItem> &items,
                       const std::function<void(size_t)> &exec_single, double *d_jac, cudaStream_t st) {
    using G = GeoA<R>;
    constexpr int kt = G::kt, a = G::a;
    if ((int)nq < kt) throw Unsupported("state narrower than the adjoint tile");
    const uint64_t low = (uint64_t(1) << G::reserve) - 1;
    const size_t n = items.size();
    // which items have a register form (checked with the tile-local map of a full tile)
    std::vector<int> ident(nq);
    for (uint32_t x = 0; x < nq; ++x) ident[x] = (int)x;
    auto fusable = [&](const AdjItem &it) {
        uint64_t b = 0;
        if (it.adj.kind == Kind::Noop) return false;
        if (!tile_bits(it.adj, b)) return false;
        const int64_t rt = reg_targets<R>(it.adj, ident);
        if (rt < 0) return false;
        int64_t pt = 0;
        if (it.diff && (pt = prod_targets(it.G, ident)) < 0) return false;
        // the step's targets (and its product's) must fit one phase's register bits
        return __builtin_popcountll((uint64_t)rt | (uint64_t)pt) <= a;
    };
    struct Piece {
        bool seg;
        size_t first;              // single item
        std::vector<size_t> take;  // segment items
    };
    std::vector<Piece> pieces;
    std::vector<char> done(n, 0);
    size_t first = 0;
    while (true) {
        while (first < n && done[first]) ++first;
        if (first >= n) break;
        if (!fusable(items[first])) {
            pieces.push_back(Piece{false, first, {}});
            done[first] = 1;
            continue;
        }
        uint64_t used = 0, blocked_any = 0, blocked_nondiag = 0;
        int ncf = 0, nitems = 0;
        std::vector<size_t> take;
        for (size_t j = first; j < n; ++j) {
            if (done[j]) continue;
            const AdjItem &it = items[j];
            const uint64_t db = dep_bits(it.adj) | (it.diff ? dep_bits(it.G) : 0);
            const bool diagonal = is_diagonal(it.adj);
            const bool blocked = (db & blocked_nondiag) || (!diagonal && (db & blocked_any));
            uint64_t b = 0;
            bool fits = !blocked && fusable(it) && tile_bits(it.adj, b);
            if (fits) {
                b |= it.diff ? dep_bits(it.G) : 0;
                fits = __builtin_popcountll(used | b | low) <= kt && (int)take.size() + 1 <= kMaxAdjItems &&
                       ncf + coef_count(it.adj) <= kMaxAdjCoefs && nitems + (it.diff ? 1 : 0) <= kMaxAdjItems;
            }
            if (fits) {
                used |= b;
                ncf += coef_count(it.adj);
                nitems += it.diff ? 1 : 0;
                take.push_back(j);
            } else {
                blocked_any |= db;
                if (!diagonal) blocked_nondiag |= db;
            }
        }
        for (size_t j : take) done[j] = 1;
        pieces.push_back(Piece{true, 0, take});
    }
    // lower every segment (records per segment, launched in order with the singles between)
    struct SegRec {
        std::vector<uint8_t> lbits, gbits;
        SegCode<R> sc;
        std::vector<PProd> prods;
        std::vector<double2> gcf;
        std::vector<double> alpha;
        std::vector<int64_t> col;
    };
    std::vector<SegRec> recs;
    for (const Piece &pc : pieces) {
        if (!pc.seg) continue;
        SegRec r;
        uint64_t used = 0;
        for (size_t j : pc.take) {
            uint64_t b = 0;
            tile_bits(items[j].adj, b);
            used |= b | (items[j].diff ? dep_bits(items[j].G) : 0);
        }
        std::vector<int> loc(nq, -1);
        uint64_t inl = used | low;
        for (uint32_t x = 0; x < nq && __builtin_popcountll(inl) < kt; ++x) inl |= uint64_t(1) << x;
        for (uint32_t x = 0; x < nq; ++x) {
            if ((inl >> x) & 1) {
                loc[x] = (int)r.lbits.size();
                r.lbits.push_back((uint8_t)x);
            } else {
                r.gbits.push_back((uint8_t)x);
            }
        }
        // phases over the items in sweep order (no reordering inside a segment: products must
        // see exactly the steps before them)
        std::vector<const GateDesc *> cur;
        std::vector<size_t> cur_items;
        uint32_t rmask = 0;
        auto close = [&]() {
            if (cur.empty()) return;
            RopHook hook = [&](size_t i, ROp &rop, const int *rpos) {
                const AdjItem &it = items[cur_items[i]];
                if (!it.diff) return;
                PProd q;
                const int item = (int)r.alpha.size();
                if (!lower_prod(it.G, loc, rpos, item, q, r.gcf)) throw Unsupported("adjoint product form");
                rop.prod = (int32_t)r.prods.size();
                r.prods.push_back(q);
                r.alpha.push_back(it.alpha);
                r.col.push_back(it.col);
            };
            lower_phase<R, G>(r.sc, rmask, cur, loc, hook);
            cur.clear();
            cur_items.clear();
            rmask = 0;
        };
        for (size_t j : pc.take) {
            const AdjItem &it = items[j];
            uint32_t need = (uint32_t)reg_targets<R>(it.adj, loc);
            if (it.diff) need |= (uint32_t)prod_targets(it.G, loc);
            if (__builtin_popcount(rmask | need) > a) close();
            rmask |= need;
            cur.push_back(&it.adj);
            cur_items.push_back(j);
        }
        close();
        recs.push_back(std::move(r));
    }
    // device copies and launches
    const size_t tile_bytes = sizeof(C<R>) << kt;
    const uint64_t ntiles = uint64_t(1) << (nq - kt);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sm_count());
    size_t max_items = 1;
    for (auto &r : recs) max_items = std::max(max_items, r.alpha.size());
    double *d_partials = nullptr;
    B200SV_CUDA(cudaMallocAsync((void **)&d_partials, max_items * grid * sizeof(double), st));
    std::vector<void *> frees{d_partials};
    struct Free {
        std::vector<void *> &p;
        cudaStream_t s;
        ~Free() {
            for (void *x : p) cudaFreeAsync(x, s);
        }
    } fr{frees, st};
    size_t si = 0;
    for (const Piece &pc : pieces) {
        if (!pc.seg) {
            exec_single(pc.first);
            continue;
        }
        SegRec &r = recs[si++];
        const size_t bph = r.sc.phases.size() * sizeof(RPhase), brop = r.sc.rops.size() * sizeof(ROp),
                     bpr = r.prods.size() * sizeof(PProd), bg = r.gcf.size() * sizeof(double2),
                     bcf = r.sc.coefs.size() * sizeof(C<R>), bal = r.alpha.size() * sizeof(double),
                     bco = r.col.size() * sizeof(int64_t);
        std::vector<unsigned char> blob(bph + brop + bpr + bg + bcf + bal + bco + 64);
        size_t off = 0;
        auto put = [&](const void *src, size_t bytes) {
            const size_t o = off;
            if (bytes) std::memcpy(blob.data() + off, src, bytes);
            off += (bytes + 15) & ~size_t(15);
            return o;
        };
        const size_t o_ph = put(r.sc.phases.data(), bph), o_rop = put(r.sc.rops.data(), brop),
                     o_pr = put(r.prods.data(), bpr), o_g = put(r.gcf.data(), bg), o_cf = put(r.sc.coefs.data(), bcf),
                     o_al = put(r.alpha.data(), bal), o_co = put(r.col.data(), bco);
        unsigned char *d_blob = nullptr;
        B200SV_CUDA(cudaMallocAsync((void **)&d_blob, std::max<size_t>(off, 16), st));
        frees.push_back(d_blob);
        B200SV_CUDA(cudaMemcpyAsync(d_blob, blob.data(), off, cudaMemcpyHostToDevice, st));
        AdjSegArgs A{};
        A.phases = reinterpret_cast<const RPhase *>(d_blob + o_ph);
        A.rops = reinterpret_cast<const ROp *>(d_blob + o_rop);
        A.prods = reinterpret_cast<const PProd *>(d_blob + o_pr);
        A.gcoefs = reinterpret_cast<const double2 *>(d_blob + o_g);
        A.coefs = d_blob + o_cf;
        A.nph = (int)r.sc.phases.size();
        A.nrop = (int)r.sc.rops.size();
        A.nprod = (int)r.prods.size();
        A.ngcoef = (int)r.gcf.size();
        A.ncoef = (int)r.sc.coefs.size();
        A.nitems = (int)r.alpha.size();
        A.ng = (int)r.gbits.size();
        std::memcpy(A.lbits, r.lbits.data(), r.lbits.size());
        std::memcpy(A.gbits, r.gbits.data(), r.gbits.size());
        const size_t smem = 4 * tile_bytes + bph + brop + bpr + bg + (size_t)A.nitems * kWarps * sizeof(double) + bcf;
        if (smem > 227 * 1024) throw Unsupported("fused adjoint segment exceeds shared memory");
        B200SV_CUDA(cudaFuncSetAttribute(k_fused_adj<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_fused_adj<R><<<grid, kFThreads, smem, st>>>(static_cast<C<R> *>(lam), static_cast<C<R> *>(bra), A, ntiles,
                                                      d_partials);
        B200SV_CUDA(cudaGetLastError());
        if (A.nitems) {
            k_adj_fused_final<<<A.nitems, 128, 0, st>>>(d_partials, (int)grid,
                                                         reinterpret_cast<const double *>(d_blob + o_al),
                                                         reinterpret_cast<const int64_t *>(d_blob + o_co), d_jac);
            B200SV_CUDA(cudaGetLastError());
        }
    }
}

}  // namespace

int fused_tile_bits(int dtype, uint32_t nq) {
    const int kt = dtype == B200SV_C64 ? Geo<float>::kt : Geo<double>::kt;
    return (int)std::min<uint32_t>(kt, nq);
}

// From one tile up: a narrow state leaves SMs idle during a segment, but one launch per
// segment instead of one per gate is still the shorter path for L2-resident states, where
// per-gate launches are bound by launch latency.
bool fused_worthwhile(int dtype, uint32_t nq) {
    return nq >= (uint32_t)(dtype == B200SV_C64 ? Geo<float>::kt : Geo<double>::kt);
}

void apply_fused(void *state, uint32_t nq, int dtype, const std::vector<GateDesc> &descs,
                 const std::function<void(const GateDesc &)> &apply_single, cudaStream_t st) {
    if (nq > 48 + 16) throw Unsupported("state too wide for the fused path");
    if (dtype == B200SV_C64) run_fused<float>(state, nq, descs, apply_single, st);
    else run_fused<double>(state, nq, descs, apply_single, st);
}

bool fused_adjoint_worthwhile(int dtype, uint32_t nq) {
    return nq >= (uint32_t)(dtype == B200SV_C64 ? GeoA<float>::kt : GeoA<double>::kt);
}

void apply_fused_adjoint(void *lambda, void *bra, uint32_t nq, int dtype, const std::vector<AdjItem> &items,
                         const std::function<void(size_t)> &exec_single, double *d_jac, cudaStream_t st) {
    if (nq > 48 + 16) throw Unsupported("state too wide for the fused path");
    if (dtype == B200SV_C64) run_fused_adjoint<float>(lambda, bra, nq, items, exec_single, d_jac, st);
    else run_fused_adjoint<double>(lambda, bra, nq, items, exec_single, d_jac, st);
}

}  // namespace b200sv
