// sv_fused.cu — one HBM pass for a run of gates on a single large state.
//
// The per-gate kernels (sv_gates.cu) read and write the whole state once per gate.
// Here consecutive gates whose wires fit in one shared-memory tile of 2^kt amplitudes
// form a segment: every CTA of a persistent grid takes tiles (the amplitudes that
// share the values of the n - kt bits outside the tile), applies all of the segment's
// gates to the tile in shared memory and writes it back.  Tiles always contain the
// lowest state bits, so a tile is a set of contiguous 128-byte (or longer) runs, and
// tiles are double-buffered: cp.async brings the next tile in while the current one
// is computed and stored.  Gate coefficients come from the same compiled GateDesc as
// the per-gate path (FP64 on the host, rounded once to the state's precision) and are
// staged in shared memory once per CTA; complex64 outputs are compensated sums
// (CAcc<float>), as in the per-gate kernels.
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
constexpr int kMaxSegOps = 96;
constexpr int kMaxSegCoefs = 2048;

// One gate in tile-local bit positions.
struct FOp {
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

struct SegArgs {
    const FOp *ops;
    const void *coefs;
    int nops, ncoef;
    int kt, ng;
    uint8_t lbits[16];  // state position of tile bit i (ascending)
    uint8_t gbits[48];  // state positions of the bits outside the tile (ascending)
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

// The op's masks and offsets (and the coefficients of one- and two-wire gates) are copied
// to registers before the group loop: the tile and the op records share shared memory, so
// without the copies every store to the tile would force them to be read again.
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

template <typename R, int K>
__device__ __forceinline__ void f_dense(C<R> *s, const FOp &op, const C<R> *cf, int kt) {
    constexpr int D = 1 << K;
    constexpr int NCR = K <= 2 ? D * D : 1;  // coefficients held in registers
    const OpRegs o = op_regs<D>(op);
    C<R> m[NCR];
#pragma unroll
    for (int i = 0; i < NCR; ++i) m[i] = cf[i];
    const uint32_t ng = 1u << (kt - o.nb);
    for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
        const uint32_t b = ins_group(g, o.low, o.nb) | o.cmask;
        C<R> v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = s[b + o.off[r]];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            CAcc<R> a;
#pragma unroll
            for (int c = 0; c < D; ++c) a.add(K <= 2 ? m[(r * D + c) % NCR] : cf[r * D + c], v[c]);
            s[b + o.off[r]] = a.get();
        }
    }
}

template <typename R, int K>
__device__ __forceinline__ void f_diag(C<R> *s, const FOp &op, const C<R> *cf, int kt) {
    constexpr int D = 1 << K;
    const OpRegs o = op_regs<D>(op);
    C<R> m[D];
#pragma unroll
    for (int r = 0; r < D; ++r) m[r] = cf[r];
    const uint32_t ng = 1u << (kt - o.nb);
    for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
        const uint32_t b = ins_group(g, o.low, o.nb) | o.cmask;
#pragma unroll
        for (int r = 0; r < D; ++r) {
            CAcc<R> a;
            a.add(m[r], s[b + o.off[r]]);
            s[b + o.off[r]] = a.get();
        }
    }
}

template <typename R>
__device__ __forceinline__ void f_swap(C<R> *s, const FOp &op, int kt) {
    const OpRegs o = op_regs<1>(op);
    const uint32_t ng = 1u << (kt - o.nb);
    const uint32_t oa = op.off[op.ra], ob = op.off[op.rb];
    for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
        const uint32_t b = ins_group(g, o.low, o.nb) | o.cmask;
        const C<R> t = s[b + oa];
        s[b + oa] = s[b + ob];
        s[b + ob] = t;
    }
}

template <typename R>
__device__ __forceinline__ void f_pair(C<R> *s, const FOp &op, const C<R> *cf, int kt) {
    const OpRegs o = op_regs<16>(op);
    const int D = 1 << op.k, ra = op.ra, rb = op.rb, rest = op.rest;
    C<R> m[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) m[i] = cf[i];
    const uint32_t ng = 1u << (kt - o.nb);
    const uint32_t oa = op.off[ra], ob = op.off[rb];  // run-time rows: read from the record, once
    for (uint32_t g = threadIdx.x; g < ng; g += blockDim.x) {
        const uint32_t b = ins_group(g, o.low, o.nb) | o.cmask;
        const C<R> va = s[b + oa], vb = s[b + ob];
        CAcc<R> x, y;
        x.add(m[0], va);
        x.add(m[1], vb);
        y.add(m[2], va);
        y.add(m[3], vb);
        s[b + oa] = x.get();
        s[b + ob] = y.get();
        if (rest) {
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                if (r >= D || r == ra || r == rb) continue;
                CAcc<R> z;
                z.add(m[4], s[b + o.off[r]]);
                s[b + o.off[r]] = z.get();
            }
        }
    }
}

template <typename R>
__device__ __forceinline__ void f_parity(C<R> *s, const FOp &op, const C<R> *cf, int kt, uint64_t tbase) {
    const uint32_t n = 1u << kt;
    const int tp = __popcll(tbase & op.pm_global) & 1;
    const uint32_t pm = op.pm_local;
    const C<R> ph0 = cf[tp], ph1 = cf[tp ^ 1];
    for (uint32_t l = threadIdx.x; l < n; l += blockDim.x) {
        CAcc<R> a;
        a.add((__popc(l & pm) & 1) ? ph1 : ph0, s[l]);
        s[l] = a.get();
    }
}

template <typename R>
__device__ void apply_fop(C<R> *s, const FOp &op, const C<R> *cf, int kt, uint64_t tbase) {
    switch (op.kind) {
    case (int)Kind::Dense:
        if (op.k == 1) f_dense<R, 1>(s, op, cf, kt);
        else if (op.k == 2) f_dense<R, 2>(s, op, cf, kt);
        else f_dense<R, 3>(s, op, cf, kt);
        break;
    case (int)Kind::Diag:
        if (op.k == 0) f_diag<R, 0>(s, op, cf, kt);
        else if (op.k == 1) f_diag<R, 1>(s, op, cf, kt);
        else f_diag<R, 2>(s, op, cf, kt);
        break;
    case (int)Kind::Swap: f_swap<R>(s, op, kt); break;
    case (int)Kind::Pair: f_pair<R>(s, op, cf, kt); break;
    case (int)Kind::Parity: f_parity<R>(s, op, cf, kt, tbase); break;
    default: break;
    }
}

__device__ __forceinline__ uint64_t deposit(uint64_t x, const uint8_t *pos, int nbits) {
    uint64_t r = 0;
    for (int i = 0; i < nbits; ++i) r |= ((x >> i) & 1u) << pos[i];
    return r;
}

// One segment over all tiles.  Shared memory: two tile buffers, the segment's ops and
// coefficients.  A tile is moved in 16-byte chunks (V amplitudes each, V = 16 / the
// amplitude size); chunk c of a thread is c = threadIdx.x + j * blockDim.x.
template <typename R>
__global__ void __launch_bounds__(kFThreads, 1) k_fused(C<R> *__restrict__ state, SegArgs a, uint64_t ntiles) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ uint8_t s_lbits[16], s_gbits[48];
    constexpr int V = 16 / (int)sizeof(C<R>);
    const uint32_t tn = 1u << a.kt;
    C<R> *const buf0 = reinterpret_cast<C<R> *>(smem_raw);
    FOp *sops = reinterpret_cast<FOp *>(smem_raw + 2 * sizeof(C<R>) * tn);
    C<R> *scf = reinterpret_cast<C<R> *>(sops + a.nops);
    if (threadIdx.x == 0) {  // constant indices keep the parameter arrays out of local memory
#pragma unroll
        for (int i = 0; i < 16; ++i) s_lbits[i] = a.lbits[i];
#pragma unroll
        for (int i = 0; i < 48; ++i) s_gbits[i] = a.gbits[i];
    }
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(a.ops);
        uint32_t *dst = reinterpret_cast<uint32_t *>(sops);
        const int words = a.nops * (int)(sizeof(FOp) / 4);
        for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
        const C<R> *cs = static_cast<const C<R> *>(a.coefs);
        for (int i = threadIdx.x; i < a.ncoef; i += blockDim.x) scf[i] = cs[i];
    }
    __syncthreads();
    // per-thread address parts: chunk c -> local amplitude c * V
    const int chunks = (int)(tn / V);
    const int per = chunks / (int)blockDim.x;  // chunks per thread (the host keeps this exact, <= 8)
    const uint64_t lo = deposit((uint64_t)threadIdx.x * V, s_lbits, a.kt);
    uint64_t hi[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) hi[j] = j < per ? deposit((uint64_t)j * blockDim.x * V, s_lbits, a.kt) : 0;

    uint64_t t = blockIdx.x;
    uint32_t cur = 0;
    if (t < ntiles) {
        const uint64_t tb = deposit(t, s_gbits, a.ng);
#pragma unroll
        for (int j = 0; j < 8; ++j)
            if (j < per) cp_async16(buf0 + (threadIdx.x + j * blockDim.x) * V, state + (tb | lo | hi[j]));
    }
    cp_async_commit();
    for (; t < ntiles; t += gridDim.x) {
        const uint64_t tnext = t + gridDim.x;
        if (tnext < ntiles) {
            const uint64_t tb = deposit(tnext, s_gbits, a.ng);
            C<R> *dst = buf0 + (cur ^ 1u) * tn;
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (j < per) cp_async16(dst + (threadIdx.x + j * blockDim.x) * V, state + (tb | lo | hi[j]));
        }
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
        C<R> *s = buf0 + cur * tn;
        const uint64_t tbase = deposit(t, s_gbits, a.ng);
        for (int o = 0; o < a.nops; ++o) {
            apply_fop<R>(s, sops[o], scf + sops[o].coef, a.kt, tbase);
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (j < per) {
                const float4 v = *reinterpret_cast<const float4 *>(s + (threadIdx.x + j * blockDim.x) * V);
                *reinterpret_cast<float4 *>(state + (tbase | lo | hi[j])) = v;
            }
        }
        __syncthreads();  // the buffer is refilled next iteration
        cur ^= 1u;
    }
    cp_async_wait0();
}

template <typename R> C<R> to_r(const cd &z) { return mk<R>((R)z.real(), (R)z.imag()); }

struct Segment {
    std::vector<uint8_t> lbits, gbits;
    uint32_t op_begin = 0, nops = 0, coef_begin = 0, ncoef = 0;
};

// Group bits (targets and controls) of a descriptor the tile kernels cover; false when
// the descriptor has to run on its own (wide dense matrices and the like).
bool tile_bits(const GateDesc &g, uint64_t &bits) {
    bits = 0;
    switch (g.kind) {
    case Kind::Noop: return true;
    case Kind::Parity: return true;
    case Kind::Dense: if (g.k < 1 || g.k > 3) return false; break;
    case Kind::Diag: if (g.k > 2) return false; break;
    case Kind::Swap: if (g.k > 3) return false; break;
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
    case Kind::Diag: return 1 << g.k;
    case Kind::Pair: return 5;
    case Kind::Parity: return 2;
    default: return 0;
    }
}

template <typename R>
FOp lower_fop(const GateDesc &g, const std::vector<int> &loc, std::vector<C<R>> &coefs) {
    FOp f{};
    f.kind = (int)g.kind;
    f.k = g.k;
    f.coef = (int32_t)coefs.size();
    if (g.kind == Kind::Parity) {
        for (int b = 0; b < 64; ++b) {
            if (!((g.pmask >> b) & 1)) continue;
            if (b < (int)loc.size() && loc[b] >= 0) f.pm_local |= 1u << loc[b];
            else f.pm_global |= uint64_t(1) << b;
        }
        coefs.push_back(to_r<R>(g.pphase[0]));
        coefs.push_back(to_r<R>(g.pphase[1]));
        return f;
    }
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
    switch (g.kind) {
    case Kind::Dense:
    case Kind::Diag:
        for (auto &z : g.m) coefs.push_back(to_r<R>(z));
        break;
    case Kind::Swap:
        f.ra = (int)g.sa;
        f.rb = (int)g.sb;
        break;
    case Kind::Pair:
        f.ra = (int)g.pa;
        f.rb = (int)g.pb;
        for (auto &z : g.m2) coefs.push_back(to_r<R>(z));
        coefs.push_back(to_r<R>(g.gamma));
        f.rest = g.gamma != cd(1.0, 0.0) ? 1 : 0;
        break;
    default: break;
    }
    return f;
}

// ---- composing consecutive gates on a few bits ------------------------------------------
// A step costs one read and one write of the tile in shared memory, which bounds complex128
// segments; gates whose bits together span at most three tile bits are multiplied into one
// 8x8 (or smaller) matrix on the host in FP64 and applied as one dense step.  The FP64 work
// per amplitude grows (8 complex products for three bits) but the FP64 pipe has room.
// complex64 steps are bound by their compensated sums (twice the FP64 cost per product), so
// complex64 composes over at most two bits: on 28 qubits a 10-layer RX RY RZ + CNOT circuit
// takes 204 ms with two bits, 248 with one, 373 with three and 791 without composition.
// The composed matrix is rounded to complex64 once, from FP64.

constexpr int kComposeBitsC64 = 2;

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

// the segment's gates with runs on at most three bits composed
std::vector<GateDesc> compose_passes(const std::vector<const GateDesc *> &in, int max_bits) {
    std::vector<GateDesc> out;
    size_t a = 0;
    while (a < in.size()) {
        uint64_t b0 = 0;
        if (!fusable(*in[a]) || !tile_bits(*in[a], b0) || __builtin_popcountll(b0) > max_bits) {
            out.push_back(*in[a++]);
            continue;
        }
        uint64_t bits = 0, b1 = 0;
        tile_bits(*in[a], bits);
        size_t b = a + 1;
        while (b < in.size() && fusable(*in[b]) && tile_bits(*in[b], b1) && __builtin_popcountll(bits | b1) <= max_bits) {
            bits |= b1;
            ++b;
        }
        if (b - a == 1) out.push_back(*in[a]);
        else out.push_back(compose(std::vector<const GateDesc *>(in.begin() + a, in.begin() + b), bits));
        a = b;
    }
    return out;
}

template <typename R>
void run_fused(void *state, uint32_t nq, const std::vector<GateDesc> &descs,
               const std::function<void(const GateDesc &)> &apply_single, cudaStream_t st) {
    const int kt = fused_tile_bits(sizeof(R) == 4 ? B200SV_C64 : B200SV_C128, nq);
    const int V = 16 / (int)sizeof(C<R>);
    // the lowest bits stay in every tile: 2^reserve contiguous amplitudes = 128 bytes
    const int reserve = sizeof(R) == 4 ? 4 : 3;
    const uint64_t low = (uint64_t(1) << reserve) - 1;
    struct Piece {
        bool seg;
        Segment s;
        size_t desc;
    };
    std::vector<Piece> pieces;
    std::vector<FOp> ops;
    std::vector<C<R>> coefs;
    size_t i = 0;
    const size_t nd = descs.size();
    while (i < nd) {
        uint64_t b = 0;
        if (descs[i].kind == Kind::Noop) { ++i; continue; }
        if (!tile_bits(descs[i], b)) {
            pieces.push_back(Piece{false, {}, i});
            ++i;
            continue;
        }
        uint64_t used = 0;
        size_t j = i;
        int nops = 0, ncf = 0;
        while (j < nd) {
            if (descs[j].kind == Kind::Noop) { ++j; continue; }
            if (!tile_bits(descs[j], b)) break;
            if (__builtin_popcountll(used | b | low) > kt) break;
            if (nops + 1 > kMaxSegOps || ncf + coef_count(descs[j]) > kMaxSegCoefs) break;
            used |= b;
            ++nops;
            ncf += coef_count(descs[j]);
            ++j;
        }
        if (j == i) {  // cannot happen for the forms above (a gate uses at most 8 tile bits); kept as a guard
            pieces.push_back(Piece{false, {}, i});
            ++i;
            continue;
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
        sg.op_begin = (uint32_t)ops.size();
        sg.coef_begin = (uint32_t)coefs.size();
        std::vector<C<R>> local;
        std::vector<const GateDesc *> seg;
        for (size_t q = i; q < j; ++q)
            if (descs[q].kind != Kind::Noop) seg.push_back(&descs[q]);
        bool composed = false;
        {
            const std::vector<GateDesc> fused = compose_passes(seg, sizeof(R) == 8 ? 3 : kComposeBitsC64);
            size_t nc = 0;
            for (auto &g : fused) nc += coef_count(g);
            if (fused.size() < seg.size() && nc <= (size_t)kMaxSegCoefs) {
                for (auto &g : fused) ops.push_back(lower_fop<R>(g, loc, local));
                composed = true;
            }
        }
        if (!composed)
            for (const GateDesc *g : seg) ops.push_back(lower_fop<R>(*g, loc, local));
        sg.nops = (uint32_t)(ops.size() - sg.op_begin);
        sg.ncoef = (uint32_t)local.size();
        coefs.insert(coefs.end(), local.begin(), local.end());
        pieces.push_back(Piece{true, sg, 0});
        i = j;
    }
    if (ops.empty()) {
        for (auto &p : pieces) apply_single(descs[p.desc]);
        return;
    }
    if ((uint32_t(1) << kt) / V % kFThreads != 0 || (uint32_t(1) << kt) / V / kFThreads > 8)
        throw Unsupported("fused tile size does not match the thread count");
    FOp *d_ops = nullptr;
    C<R> *d_cf = nullptr;
    B200SV_CUDA(cudaMallocAsync((void **)&d_ops, ops.size() * sizeof(FOp), st));
    B200SV_CUDA(cudaMallocAsync((void **)&d_cf, std::max<size_t>(1, coefs.size()) * sizeof(C<R>), st));
    struct Free {
        void *a, *b;
        cudaStream_t s;
        ~Free() {
            cudaFreeAsync(a, s);
            cudaFreeAsync(b, s);
        }
    } fr{d_ops, d_cf, st};
    B200SV_CUDA(cudaMemcpyAsync(d_ops, ops.data(), ops.size() * sizeof(FOp), cudaMemcpyHostToDevice, st));
    if (!coefs.empty())
        B200SV_CUDA(cudaMemcpyAsync(d_cf, coefs.data(), coefs.size() * sizeof(C<R>), cudaMemcpyHostToDevice, st));
    const size_t tile_bytes = sizeof(C<R>) << kt;
    const size_t smem_max = 2 * tile_bytes + kMaxSegOps * sizeof(FOp) + kMaxSegCoefs * sizeof(C<R>);
    B200SV_CUDA(cudaFuncSetAttribute(k_fused<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    const uint64_t ntiles = uint64_t(1) << (nq - kt);
    const unsigned grid = (unsigned)std::min<uint64_t>(ntiles, (uint64_t)sm_count());
    for (const Piece &p : pieces) {
        if (!p.seg) {
            apply_single(descs[p.desc]);
            continue;
        }
        SegArgs a{};
        a.ops = d_ops + p.s.op_begin;
        a.coefs = d_cf + p.s.coef_begin;
        a.nops = (int)p.s.nops;
        a.ncoef = (int)p.s.ncoef;
        a.kt = kt;
        a.ng = (int)p.s.gbits.size();
        std::memcpy(a.lbits, p.s.lbits.data(), p.s.lbits.size());
        std::memcpy(a.gbits, p.s.gbits.data(), p.s.gbits.size());
        const size_t smem = 2 * tile_bytes + p.s.nops * sizeof(FOp) + p.s.ncoef * sizeof(C<R>);
        k_fused<R><<<grid, kFThreads, smem, st>>>(static_cast<C<R> *>(state), a, ntiles);
        B200SV_CUDA(cudaGetLastError());
    }
}

}  // namespace

int fused_tile_bits(int dtype, uint32_t nq) {
    const int kt = dtype == B200SV_C64 ? 13 : 12;
    return (int)std::min<uint32_t>(kt, nq);
}

// Below 21 qubits (2^8 / 2^9 tiles) a segment has too few tiles to fill 148 SMs and one
// launch per gate is faster: on a 200-gate random sweep at 20 qubits complex128, 1.5 ms per
// gate launch against 3.9 ms fused; from 21 qubits on (L2-resident or not) the fused path
// wins on deep circuits (a 10-layer RX RY RZ + CNOT circuit: 4.2 vs 7.8 ms at 21 qubits,
// 89 vs 334 ms at 26).
bool fused_worthwhile(int dtype, uint32_t nq) {
    return nq >= (uint32_t)fused_tile_bits(dtype, nq) + (dtype == B200SV_C64 ? 8 : 9);
}

void apply_fused(void *state, uint32_t nq, int dtype, const std::vector<GateDesc> &descs,
                 const std::function<void(const GateDesc &)> &apply_single, cudaStream_t st) {
    if (nq > 48 + 16) throw Unsupported("state too wide for the fused path");
    if (dtype == B200SV_C64) run_fused<float>(state, nq, descs, apply_single, st);
    else run_fused<double>(state, nq, descs, apply_single, st);
}

}  // namespace b200sv
