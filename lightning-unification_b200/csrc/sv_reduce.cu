// sv_reduce.cu — read-only FP64 reductions over a state vector.
//
// The reference computes every expectation value by copying the state, applying
// the observable and taking innerProdC (LQ/measurements/MeasurementsLQubit.hpp:145-180,
// :248-265; LQ/utils/LinearAlgebra.hpp:151-213): three full passes per term.
// Here Pauli words are evaluated in read-only passes (diagonal words together through a
// Walsh-Hadamard transform per tile, words with nearby X masks together, each distant X mask
// in a pass over its amplitude pairs), a Hermitian matrix as v^dagger M v per group, and the
// adjoint method's -2 Im<H lambda| G |mu> (LQ/algorithms/AdjointJacobianLQubit.hpp:68-77,
// :301-323) without materialising G|mu>.  All accumulators are FP64 (complex64
// amplitudes are widened on load) and every reduction is two-pass with a fixed
// association order, so results are reproducible.
#include <algorithm>
#include <vector>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr int kRT = 256;  // reduction block size

int red_blocks(uint64_t work) {
    uint64_t b = (work + kRT * 4 - 1) / (kRT * 4);
    b = std::max<uint64_t>(1, std::min<uint64_t>(b, kMaxRedBlocks));
    return (int)b;
}

// out[v * stride] = alpha * sum_b partials[v * nb + b]  (one block per value)
__global__ void k_finalize(const double *__restrict__ partials, int nb, double *__restrict__ out,
                           int stride, double alpha) {
    __shared__ double sm[32];
    const int v = blockIdx.x;
    double s[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s[0] += partials[(size_t)v * nb + b];
    block_reduce<1>(s, sm);
    if (threadIdx.x == 0) out[(size_t)v * stride] = alpha * s[0];
}

void finalize(const double *partials, int nb, int nv, double *out, int stride, double alpha,
              cudaStream_t st) {
    k_finalize<<<nv, 128, 0, st>>>(partials, nb, out, stride, alpha);
    B200SV_CUDA(cudaGetLastError());
}

template <typename R>
__global__ void __launch_bounds__(kRT) k_norm2(const C<R> *__restrict__ a, uint64_t n, double *partials) {
    __shared__ double sm[32];
    double acc[1] = {0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 z = widen<R>(a[i]);
        acc[0] += z.x * z.x + z.y * z.y;
    }
    block_reduce<1>(acc, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

template <typename R>
__global__ void __launch_bounds__(kRT) k_inner(const C<R> *__restrict__ b, const C<R> *__restrict__ k,
                                               uint64_t n, double *partials) {
    __shared__ double sm[64];
    double acc[2] = {0.0, 0.0};
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 x = widen<R>(b[i]), y = widen<R>(k[i]);
        acc[0] += x.x * y.x + x.y * y.y;  // Re conj(x) y
        acc[1] += x.x * y.y - x.y * y.x;  // Im conj(x) y
    }
    block_reduce<2>(acc, sm);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = acc[0];
        partials[gridDim.x + blockIdx.x] = acc[1];
    }
}

// ---- generator products ----------------------------------------------------
// A generator acts on a group of 2^k rows (Dense k<=2, Diag k<=2, Pair k in {1,2,4})
// or on single amplitudes by parity; w = G v is formed in registers.
template <typename R> struct GenP {
    int kind, k;
    Insert ins;
    uint64_t ngroups;
    uint64_t off[16];
    C<R> m[16];     // Dense 4x4 (k<=2) or Diag phases
    C<R> m2[4], gamma;
    int pa, pb;
    uint64_t pmask;
    C<R> pph[2];
};
template <typename R> struct Bras {
    const C<R> *p[16];
};
// Row r of a group takes part in <bra|G|ket>: every row except, for the pair form with a zero
// gamma (the excitation generators), the rows outside the 2x2 block.
template <typename R, int KIND> __device__ __forceinline__ bool gen_row_used(const GenP<R> &p, int r) {
    if constexpr (KIND == (int)Kind::Pair)
        return r == p.pa || r == p.pb || p.gamma.x != 0 || p.gamma.y != 0;
    return true;
}

// w = G v over one group, G's form (KIND) and width (K; the group has 2^K rows, one amplitude
// for the parity form) fixed at compile time so the group stays in registers.
template <typename R, int KIND, int K>
__device__ __forceinline__ void gen_apply(const GenP<R> &p, uint64_t g, const C<R> *__restrict__ ket,
                                          uint64_t &base, double2 (&w)[1 << K]) {
    constexpr int D = 1 << K;
    if constexpr (KIND == (int)Kind::Parity) {
        base = g;
        const double2 v = widen<R>(ket[g]);
        const C<R> f = p.pph[__popcll(g & p.pmask) & 1];
        w[0] = make_double2(f.x * v.x - f.y * v.y, f.x * v.y + f.y * v.x);
        return;
    } else {
        base = p.ins(g);
        double2 v[D];
#pragma unroll
        for (int r = 0; r < D; ++r)
            v[r] = gen_row_used<R, KIND>(p, r) ? widen<R>(ket[base + p.off[r]]) : make_double2(0, 0);
        if constexpr (KIND == (int)Kind::Dense) {
#pragma unroll
            for (int r = 0; r < D; ++r) {
                double re = 0, im = 0;
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    const double mr = p.m[r * D + c].x, mi = p.m[r * D + c].y;
                    re += mr * v[c].x - mi * v[c].y;
                    im += mr * v[c].y + mi * v[c].x;
                }
                w[r] = make_double2(re, im);
            }
        } else if constexpr (KIND == (int)Kind::Diag) {
#pragma unroll
            for (int r = 0; r < D; ++r) {
                const double mr = p.m[r].x, mi = p.m[r].y;
                w[r] = make_double2(mr * v[r].x - mi * v[r].y, mr * v[r].y + mi * v[r].x);
            }
        } else {  // Pair: 2x2 block on rows pa, pb, gamma on the others
            // rows pa, pb picked by masked sums: a select the compiler could turn back into a
            // run-time array index would put v in local memory
            double2 va = make_double2(0, 0), vb = make_double2(0, 0);
#pragma unroll
            for (int r = 0; r < D; ++r) {
                const double sa = r == p.pa ? 1.0 : 0.0, sb = r == p.pb ? 1.0 : 0.0;
                va.x = fma(sa, v[r].x, va.x);
                va.y = fma(sa, v[r].y, va.y);
                vb.x = fma(sb, v[r].x, vb.x);
                vb.y = fma(sb, v[r].y, vb.y);
            }
            const C<R> m0 = p.m2[0], m1 = p.m2[1], m2 = p.m2[2], m3 = p.m2[3];
            const double2 wa = make_double2(m0.x * va.x - m0.y * va.y + m1.x * vb.x - m1.y * vb.y,
                                            m0.x * va.y + m0.y * va.x + m1.x * vb.y + m1.y * vb.x);
            const double2 wb = make_double2(m2.x * va.x - m2.y * va.y + m3.x * vb.x - m3.y * vb.y,
                                            m2.x * va.y + m2.y * va.x + m3.x * vb.y + m3.y * vb.x);
            const double gr = p.gamma.x, gi = p.gamma.y;
#pragma unroll
            for (int r = 0; r < D; ++r)
                w[r] = r == p.pa ? wa
                     : r == p.pb ? wb
                                 : make_double2(gr * v[r].x - gi * v[r].y, gr * v[r].y + gi * v[r].x);
        }
    }
}

// Both components of <bra|G|ket> for one bra: partials[0..nb) = Re, [nb..2nb) = Im.
template <typename R, int KIND, int K>
__global__ void __launch_bounds__(kRT) k_gen_inner_c(const C<R> *__restrict__ bra, const C<R> *__restrict__ ket,
                                                     GenP<R> p, double *partials) {
    __shared__ double sm[2 * 32];
    constexpr int D = 1 << K;
    double acc[2] = {0.0, 0.0};
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t base;
        double2 w[D];
        gen_apply<R, KIND, K>(p, g, ket, base, w);
#pragma unroll
        for (int r = 0; r < D; ++r) {
            if (!gen_row_used<R, KIND>(p, r)) continue;
            const uint64_t idx = KIND == (int)Kind::Parity ? base : base + p.off[r];
            const double2 b = widen<R>(bra[idx]);
            acc[0] += b.x * w[r].x + b.y * w[r].y;  // Re conj(b) w
            acc[1] += b.x * w[r].y - b.y * w[r].x;  // Im conj(b) w
        }
    }
    block_reduce<2>(acc, sm);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = acc[0];
        partials[gridDim.x + blockIdx.x] = acc[1];
    }
}

// With `fin` set, the last block to finish also forms the results (out[o * stride] = alpha *
// the sum of partials[o][*], per bra a warp summing in a fixed order) and rearms fin->count,
// which saves the separate finalize launch in the adjoint sweep's per-parameter loop.
struct GenFinal {
    unsigned int *count;  // zero before the launch; zero again after it
    double *out;
    int stride;
    double alpha;
};
template <typename R, int NB, int KIND, int K>
__global__ void __launch_bounds__(kRT) k_gen_inner(Bras<R> bras, int nbra, const C<R> *__restrict__ ket,
                                                   GenP<R> p, double *partials, GenFinal fin) {
    __shared__ double sm[NB * 32];
    constexpr int D = 1 << K;
    double acc[NB];
#pragma unroll
    for (int o = 0; o < NB; ++o) acc[o] = 0.0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t base;
        double2 w[D];
        gen_apply<R, KIND, K>(p, g, ket, base, w);
#pragma unroll
        for (int r = 0; r < D; ++r) {
            if (!gen_row_used<R, KIND>(p, r)) continue;
            const uint64_t idx = KIND == (int)Kind::Parity ? base : base + p.off[r];
#pragma unroll
            for (int o = 0; o < NB; ++o) {
                if (o < nbra) {
                    const double2 b = widen<R>(bras.p[o][idx]);
                    acc[o] += b.x * w[r].y - b.y * w[r].x;  // Im conj(b) w
                }
            }
        }
    }
    block_reduce<NB>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int o = 0; o < NB; ++o)
            if (o < nbra) partials[(size_t)o * gridDim.x + blockIdx.x] = acc[o];
    }
    if (fin.count == nullptr) return;
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();  // this block's partials before its arrival
        last = atomicAdd(fin.count, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = warp; o < nbra; o += (int)(blockDim.x >> 5)) {
        double v = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) v += __ldcg(&partials[(size_t)o * gridDim.x + b]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) fin.out[(size_t)o * fin.stride] = fin.alpha * v;
    }
    if (threadIdx.x == 0) *fin.count = 0u;
}

// launchers of the two inner-product kernels for one generator form (with_gen_form)
template <typename R> struct GoGenC {
    int nb;
    cudaStream_t st;
    const C<R> *b, *k;
    const GenP<R> &p;
    double *partials;
    template <int KIND, int K> void go() const { k_gen_inner_c<R, KIND, K><<<nb, kRT, 0, st>>>(b, k, p, partials); }
};
template <typename R> struct GoGen {
    int nb, nbra;
    cudaStream_t st;
    const Bras<R> &B;
    const C<R> *k;
    const GenP<R> &p;
    double *partials;
    GenFinal fin;
    template <int KIND, int K> void go() const {
        if (nbra == 1) k_gen_inner<R, 1, KIND, K><<<nb, kRT, 0, st>>>(B, nbra, k, p, partials, fin);
        else if (nbra <= 4) k_gen_inner<R, 4, KIND, K><<<nb, kRT, 0, st>>>(B, nbra, k, p, partials, fin);
        else k_gen_inner<R, 16, KIND, K><<<nb, kRT, 0, st>>>(B, nbra, k, p, partials, fin);
    }
};

// Call f.template go<KIND, K>() for the generator form of p (the forms and widths
// compile_generator produces).
template <typename R, typename F> void with_gen_form(const GenP<R> &p, const F &f) {
    switch (p.kind) {
    case (int)Kind::Parity: f.template go<(int)Kind::Parity, 0>(); return;
    case (int)Kind::Dense:
        if (p.k == 1) f.template go<(int)Kind::Dense, 1>();
        else f.template go<(int)Kind::Dense, 2>();
        return;
    case (int)Kind::Diag:
        if (p.k == 0) f.template go<(int)Kind::Diag, 0>();
        else if (p.k == 1) f.template go<(int)Kind::Diag, 1>();
        else f.template go<(int)Kind::Diag, 2>();
        return;
    case (int)Kind::Pair:
        if (p.k == 1) f.template go<(int)Kind::Pair, 1>();
        else if (p.k == 2) f.template go<(int)Kind::Pair, 2>();
        else if (p.k == 4) f.template go<(int)Kind::Pair, 4>();
        else throw Unsupported("generator pair form on 1, 2 or 4 wires");
        return;
    default: throw Unsupported("generator form not supported in the inner product");
    }
}

// ---- Hermitian sandwich ------------------------------------------------------
template <typename R> struct DenseEvP {
    Insert ins;
    uint64_t ngroups;
    uint64_t off[16];
    int k;
};
// K is a template parameter so the group's amplitudes stay in registers (a run-time 2^k
// indexed its array dynamically and put it in local memory)
template <typename R, int K>
__global__ void __launch_bounds__(kRT) k_dense_ev(const C<R> *__restrict__ a, DenseEvP<R> p,
                                                  const C<R> *__restrict__ m, double *partials) {
    __shared__ double sm[32];
    constexpr int D = 1 << K;
    double acc[1] = {0.0};
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g);
        double2 v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = widen<R>(a[base + p.off[r]]);
#pragma unroll
        for (int r = 0; r < D; ++r) {
            double re = 0, im = 0;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                const C<R> x = __ldg(&m[r * D + c]);
                re += (double)x.x * v[c].x - (double)x.y * v[c].y;
                im += (double)x.x * v[c].y + (double)x.y * v[c].x;
            }
            acc[0] += v[r].x * re + v[r].y * im;  // Re conj(v_r) (M v)_r
        }
    }
    block_reduce<1>(acc, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

// ---- marginal probabilities --------------------------------------------------
struct ProbsP {
    Insert others;        // inserts zeros at the measured bits
    uint64_t nothers;
    uint64_t binmask[64];  // bin bit (k-1-j) -> state bit bits[j]
    int k;
    uint64_t nbins;
};
__device__ __forceinline__ uint64_t deposit_bin(const ProbsP &p, uint64_t m) {
    uint64_t o = 0;
    for (int j = 0; j < p.k; ++j)
        if (m & (uint64_t(1) << (p.k - 1 - j))) o |= p.binmask[j];
    return o;
}
// 8 bins per block row (blockIdx.y), blocks along x split the other indices
template <typename R>
__global__ void __launch_bounds__(kRT) k_probs_hist(const C<R> *__restrict__ a, ProbsP p, double *partials) {
    __shared__ double sm[8 * 32];
    double acc[8];
    uint64_t bo[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        acc[q] = 0.0;
        const uint64_t m = (uint64_t)blockIdx.y * 8 + q;
        bo[q] = m < p.nbins ? deposit_bin(p, m) : 0;
    }
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < p.nothers;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.others(r);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if ((uint64_t)blockIdx.y * 8 + q < p.nbins) {
                const double2 z = widen<R>(a[base | bo[q]]);
                acc[q] += z.x * z.x + z.y * z.y;
            }
        }
    }
    block_reduce<8>(acc, sm);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 8; ++q) {
            const uint64_t m = (uint64_t)blockIdx.y * 8 + q;
            if (m < p.nbins) partials[m * gridDim.x + blockIdx.x] = acc[q];
        }
    }
}
template <typename R>
__global__ void __launch_bounds__(kRT) k_probs_perbin(const C<R> *__restrict__ a, ProbsP p, double *out) {
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < p.nbins;
         m += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t bo = deposit_bin(p, m);
        double s = 0.0;
        for (uint64_t r = 0; r < p.nothers; ++r) {
            const double2 z = widen<R>(a[p.others(r) | bo]);
            s += z.x * z.x + z.y * z.y;
        }
        out[m] = s;
    }
}
template <typename R>
__global__ void __launch_bounds__(kRT) k_probs_all(const C<R> *__restrict__ a, uint64_t n, double *out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 z = widen<R>(a[i]);
        out[i] = z.x * z.x + z.y * z.y;
    }
}

// ---- elementwise -------------------------------------------------------------
template <typename R> __global__ void k_set_one(C<R> *a, uint64_t idx) { a[idx] = mk<R>(1, 0); }

template <typename R>
__global__ void __launch_bounds__(kRT) k_axpy_pauli(C<R> *__restrict__ acc, const C<R> *__restrict__ x, uint64_t n,
                                                    uint64_t xmask, uint64_t zmask, int ny, double cr) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 v = widen<R>(x[i]);
        double fr = (__popcll(i & zmask) & 1) ? -cr : cr, fi = 0.0;
        switch (ny & 3) {  // multiply by i^ny
        case 1: fi = fr; fr = 0; break;
        case 2: fr = -fr; break;
        case 3: fi = -fr; fr = 0; break;
        default: break;
        }
        const uint64_t j = i ^ xmask;
        const double2 a = widen<R>(acc[j]);
        acc[j] = mk<R>((R)(a.x + fr * v.x - fi * v.y), (R)(a.y + fr * v.y + fi * v.x));
    }
}
template <typename R>
__global__ void __launch_bounds__(kRT) k_axpy(C<R> *__restrict__ acc, const C<R> *__restrict__ x, uint64_t n, double c) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double2 v = widen<R>(x[i]), a = widen<R>(acc[i]);
        acc[i] = mk<R>((R)(a.x + c * v.x), (R)(a.y + c * v.y));
    }
}

dim3 ew_grid(uint64_t n) {
    uint64_t b = (n + kRT - 1) / kRT;
    const uint64_t cap = uint64_t(sm_count()) * 16;
    return dim3((unsigned)std::max<uint64_t>(1, std::min(b, cap)));
}

Insert insert_of(std::vector<uint32_t> bits) {
    std::sort(bits.begin(), bits.end());
    Insert ins{};
    ins.nb = (int)bits.size();
    if (ins.nb > kMaxInsert) throw Unsupported("too many inserted bits");
    for (int j = 0; j < ins.nb; ++j) ins.low[j] = (uint64_t(1) << bits[j]) - 1;
    return ins;
}

template <typename R> C<R> cvt(const cd &z) { return mk<R>((R)z.real(), (R)z.imag()); }

}  // namespace

template <typename R>
void reduce_norm2(const void *a, uint32_t nq, double *partials, double *out, cudaStream_t st) {
    const uint64_t n = uint64_t(1) << nq;
    const int nb = red_blocks(n);
    k_norm2<R><<<nb, kRT, 0, st>>>(static_cast<const C<R> *>(a), n, partials);
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, 1, out, 1, 1.0, st);
}

template <typename R>
void reduce_inner(const void *bra, const void *ket, uint32_t nq, double *partials, double *out,
                  cudaStream_t st) {
    const uint64_t n = uint64_t(1) << nq;
    const int nb = red_blocks(n);
    k_inner<R><<<nb, kRT, 0, st>>>(static_cast<const C<R> *>(bra), static_cast<const C<R> *>(ket), n, partials);
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, 2, out, 1, 1.0, st);
}

// ---- Pauli words sharing an X mask -----------------------------------------
// P|i> = i^ny (-1)^popcount(i & zmask) |i ^ xmask>  (zmask covers Z and Y factors)
struct PauliGroupP {
    uint64_t xmask, hb_low;  // hb_low: (1 << highest X bit) - 1, or 0 when xmask == 0
    uint64_t npairs;
    int nterms;
    int norm;               // also accumulate <psi|psi> (after the words)
    uint64_t zmask[32];
    double cr[32], ci[32];  // Re(i^ny z) = cr Re z + ci Im z
};
template <typename R, int NT>
__global__ void __launch_bounds__(kRT) k_pauli(const C<R> *__restrict__ a, PauliGroupP p, double *partials) {
    __shared__ double sm[(NT + 1) * 32];
    double acc[NT + 1];
#pragma unroll
    for (int t = 0; t <= NT; ++t) acc[t] = 0.0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        if (p.xmask == 0) {
            const double2 z = widen<R>(a[g]);
            const double pr = z.x * z.x + z.y * z.y;
#pragma unroll
            for (int t = 0; t < NT; ++t)
                if (t < p.nterms) acc[t] += (__popcll(g & p.zmask[t]) & 1) ? -pr : pr;
            acc[NT] += pr;
        } else {
            const uint64_t lo = g & p.hb_low;
            const uint64_t i = ((g ^ lo) << 1) | lo;  // highest X bit cleared
            const uint64_t j = i ^ p.xmask;
            const double2 vi = widen<R>(a[i]), vj = widen<R>(a[j]);
            const double zr = 2.0 * (vj.x * vi.x + vj.y * vi.y);  // 2 conj(vj) vi: both ends of the pair
            const double zi = 2.0 * (vj.x * vi.y - vj.y * vi.x);
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                if (t < p.nterms) {
                    const double r = fma(p.cr[t], zr, p.ci[t] * zi);
                    acc[t] += (__popcll(i & p.zmask[t]) & 1) ? -r : r;
                }
            }
            acc[NT] += vi.x * vi.x + vi.y * vi.y + vj.x * vj.x + vj.y * vj.y;
        }
    }
    block_reduce<NT + 1>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < NT; ++t)
            if (t < p.nterms) partials[(size_t)t * gridDim.x + blockIdx.x] = acc[t];
        if (p.norm) partials[(size_t)p.nterms * gridDim.x + blockIdx.x] = acc[NT];
    }
}

// ---- Pauli words with different X masks, one pass -----------------------------
// <psi|P|psi> = sum_i conj(psi_i) i^ny (-1)^popcount((i ^ x) & zmask) psi_(i ^ x), summed over
// every i (each pair of amplitudes is visited from both ends).  Words come sorted by X mask;
// a word whose mask differs from the previous word's loads its partner amplitude, the others
// reuse it.  Per word the i^ny phase is a precomputed pair (cr, ci) applied to conj(v) u and
// the sign a parity flip, so the inner step is branch-free; states of up to 32 qubits use
// 32-bit index arithmetic.
struct PauliMultiP {
    uint64_t n;
    int nterms;
    uint64_t xmask[32];
    uint64_t zmask[32];
    double cr[32], ci[32];  // Re(i^ny z) = cr Re z + ci Im z
    int newx[32];           // 1: this word's X mask differs from the previous word's
};
template <typename R, int NT, typename I>
__global__ void __launch_bounds__(kRT) k_pauli_multi(const C<R> *__restrict__ a, PauliMultiP p, double *partials) {
    // U amplitudes per thread and trip, so U loads (and U partner loads per X mask) are in
    // flight together
    constexpr int U = 4;
    __shared__ double sm[NT * 32];
    double acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t] = 0.0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i0 < p.n; i0 += U * stride) {
        I i[U];
        bool in[U];
        double2 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            in[u] = i0 + u * stride < p.n;
            i[u] = (I)(in[u] ? i0 + u * stride : i0);
            v[u] = widen<R>(a[i[u]]);
        }
        double zr[U], zi[U];  // conj(v) * partner
#pragma unroll
        for (int u = 0; u < U; ++u) zr[u] = zi[u] = 0.0;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
            if (t < p.nterms) {
                const I x = (I)p.xmask[t], z = (I)p.zmask[t];
                if (p.newx[t]) {
                    double2 w[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) w[u] = x ? widen<R>(a[i[u] ^ x]) : v[u];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        zr[u] = v[u].x * w[u].x + v[u].y * w[u].y;
                        zi[u] = v[u].x * w[u].y - v[u].y * w[u].x;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double r = fma(p.cr[t], zr[u], p.ci[t] * zi[u]);
                    const I m = (i[u] ^ x) & z;
                    const int odd = (sizeof(I) == 8 ? __popcll((uint64_t)m) : __popc((uint32_t)m)) & 1;
                    acc[t] += in[u] ? (odd ? -r : r) : 0.0;
                }
            }
        }
    }
    block_reduce<NT>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < NT; ++t)
            if (t < p.nterms) partials[(size_t)t * gridDim.x + blockIdx.x] = acc[t];
    }
}

template <typename R>
void reduce_pauli_group(const void *psi, uint32_t nq, const PauliWord *terms, int nterms, double *partials,
                        double *out, cudaStream_t st, bool with_norm) {
    if (nterms <= 0) return;
    if (nterms > 32) throw ArgError("at most 32 Pauli words per group");
    PauliGroupP p{};
    p.xmask = terms[0].xmask;
    p.nterms = nterms;
    p.norm = with_norm ? 1 : 0;
    for (int t = 0; t < nterms; ++t) {
        if (terms[t].xmask != p.xmask) throw ArgError("Pauli group with mixed X masks");
        p.zmask[t] = terms[t].zmask;
        const int ny = terms[t].ny & 3;  // Re(i^ny z): z.re, -z.im, -z.re, z.im
        p.cr[t] = ny == 0 ? 1.0 : ny == 2 ? -1.0 : 0.0;
        p.ci[t] = ny == 1 ? -1.0 : ny == 3 ? 1.0 : 0.0;
    }
    const uint64_t n = uint64_t(1) << nq;
    if (p.xmask) {
        int hb = 63 - __builtin_clzll(p.xmask);
        p.hb_low = (uint64_t(1) << hb) - 1;
        p.npairs = n / 2;
    } else {
        p.hb_low = 0;
        p.npairs = n;
    }
    const int nb = red_blocks(p.npairs);
    const C<R> *a = static_cast<const C<R> *>(psi);
    if (nterms == 1) k_pauli<R, 1><<<nb, kRT, 0, st>>>(a, p, partials);
    else if (nterms <= 8) k_pauli<R, 8><<<nb, kRT, 0, st>>>(a, p, partials);
    else k_pauli<R, 32><<<nb, kRT, 0, st>>>(a, p, partials);
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, nterms + (with_norm ? 1 : 0), out, 1, 1.0, st);
}

// ---- Pauli words with wide X masks, one pass over tiles -------------------------------------
// A word whose X mask reaches beyond the shared passes' partner distance costs one read of
// the state as a pair pass.  A group of words whose X bits, together with the lowest state
// bits, fit in the tile bits is evaluated per tile instead: a tile is the 4096 (complex128) or
// 8192 (complex64) amplitudes that share the values of the other bits, 64 KiB staged in shared
// memory, so the group reads the state once.  Tile element r = t + 256 j is thread t's register j
// (16 or 32 registers).
//
// For P = i^ny X^x Z^z the expectation value is sum_k Re(conj(psi_(k^x)) i^ny (-1)^(k.z) psi_k),
// and because P is Hermitian the terms of k and k^x have equal real parts, so either member
// of a pair may stand for it (counted twice).  A thread takes its register element as k and
// reads the partner from shared memory, for one member of each pair:
//  * x reaches a register bit (tile bits 8 and up): the registers j whose copy of the highest
//    such bit is 0 — the same half of the registers in every thread;
//  * x lies in the thread bits only: registers j with (j & 1) equal to the thread's bit under
//    the highest bit of x — a pair's two owners differ in that bit, so each pair is taken once,
//    and every thread takes half its registers.
// Words sharing an X mask form runs of up to 4 that share the partner read and the products.
constexpr int kPTileMaxBits = 13;
constexpr int kPTileThreads = 256;
constexpr int kPTileMaxWords = 32;
constexpr int kPTileLowBits[2] = {4, 3};  // state bits always in the tile: 128-byte runs (c64, c128)
// tile shape per precision: 64 KiB of amplitudes, 8 thread bits and 4 (complex128) or 5
// (complex64) register bits
template <typename R> struct PTile {
    static constexpr int bits = sizeof(R) == 4 ? 13 : 12;
    static constexpr int per = (1 << bits) / kPTileThreads;  // registers a thread
    static constexpr int rbits = bits - 8;
};
struct PauliTiledP {
    uint64_t ntiles;
    int nterms, ng, nruns;
    uint8_t lbits[kPTileMaxBits];       // state position of tile bit b (ascending)
    uint8_t gbits[52];                  // state positions of the other bits (ascending)
    uint8_t run_begin[kPTileMaxWords + 1];
    uint32_t xl[kPTileMaxWords];        // tile-local X mask of each run
    uint32_t zl[kPTileMaxWords];        // tile-local Z mask of each word
    uint64_t zg[kPTileMaxWords];        // Z mask outside the tile (state positions) of each word
    uint8_t ny[kPTileMaxWords];         // number of Y factors mod 4 of each word
    uint8_t run_kinds[kPTileMaxWords];  // bit 0: a word of the run has even ny, bit 1: odd
};
// parity of bit b of the register index j, as a table over the 32 registers j
__constant__ const uint32_t kRegParity[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};
__device__ __forceinline__ uint64_t deposit_bits_u8(uint64_t x, const uint8_t *pos, int nbits) {
    uint64_t r = 0;
    for (int i = 0; i < nbits; ++i) r |= ((x >> i) & 1u) << pos[i];
    return r;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Per word, packed once per block: bits 0-7 the Z mask on the thread bits, bit 8 the word takes
// Im (odd ny), bit 9 the i^ny factor is negative (ny = 1, 2); beside it the parity of (j & Z)
// over the registers j as a 32-bit table.  Per run: bits 0-12 the tile-local X mask, 13-18 the
// first word, 19-21 the number of words, 22-23 which parts its words take (bit 0 Re, bit 1 Im).
__device__ __forceinline__ uint32_t tiled_word_bits(uint32_t zl, int ny) {
    return (zl & 255u) | ((uint32_t)(ny & 1) << 8) | ((uint32_t)(ny == 1 || ny == 2) << 9);
}
__device__ __forceinline__ uint32_t tiled_reg_parity(uint32_t zl) {
    uint32_t m = 0;
#pragma unroll
    for (int b = 0; b < 5; ++b)
        if ((zl >> (8 + b)) & 1) m ^= kRegParity[b];
    return m;
}

// One run of words over a tile.  NW words (1, 2 or 4; a run of 3 carries a fourth word whose
// value is dropped), KIND which part of conj(partner) own they take (0: Re, 1: Im, 2: each word
// its own), TB the highest register bit of the X mask (-1: the mask lies in the thread bits).
// Every branch on these is resolved at compile time, so the inner step is a shared-memory
// load, the product and one signed add per word.  The run's sums go, signed, into the warp's
// accumulators.
template <typename R, int NW, int KIND, int TB>
__device__ __forceinline__ void tiled_run(const C<R> *tile, const C<R> (&v)[PTile<R>::per], int tid, uint32_t xl,
                                          int w0, int nw, const uint32_t *s_word, const uint32_t *s_jpar,
                                          uint32_t tmask, double *s_acc_warp) {
    constexpr int PER = PTile<R>::per;
    uint32_t jpar[NW];
    bool im[NW];
    double sg[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const int t = w0 + (w < nw ? w : nw - 1);
        const uint32_t wb = s_word[t];
        jpar[w] = s_jpar[t];
        im[w] = (wb >> 8) & 1u;
        const int odd = (__popc(tid & wb & 255u) + (tmask >> t) + (wb >> 9)) & 1;
        sg[w] = odd ? -2.0 : 2.0;  // 2: each pair is taken once for both of its terms
    }
    double acc[2][NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) acc[0][w] = acc[1][w] = 0.0;
    auto step = [&](const double2 vi, const double2 vj, int jbit_pos, const uint32_t (&jp)[NW], int half) {
        double zr = 0.0, zi = 0.0;
        if (KIND != 1) zr = fma(vj.x, vi.x, vj.y * vi.y);
        if (KIND != 0) zi = fma(vj.x, vi.y, -(vj.y * vi.x));
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const double val = KIND == 0 ? zr : KIND == 1 ? zi : (im[w] ? zi : zr);
            acc[half][w] += ((jp[w] >> jbit_pos) & 1u) ? -val : val;
        }
    };
    if constexpr (TB >= 0) {
        // registers j with bit TB clear; partner in register j ^ xj of thread tid ^ (xl & 255)
        const C<R> *pb = tile + (tid ^ (xl & 255u));
        const uint32_t xj = xl >> 8;
        int k = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            if (j & (1 << TB)) continue;
            // complex64 (32 registers of the tile a thread): the own element is read back from
            // shared memory, so the tile's registers are free once it is stored
            C<R> own;
            if constexpr (sizeof(R) == 4) own = tile[tid + (j << 8)];
            else own = v[j];
            step(widen<R>(own), widen<R>(pb[((uint32_t)j ^ xj) << 8]), j, jpar, (k++) & 1);
        }
    } else {
        // registers j = 2m + hb (own element read back from shared memory); partner in the same
        // register of thread tid ^ xl
        const int hb = (tid >> (31 - __clz(xl))) & 1;
        const C<R> *po = tile + tid + (hb << 8);
        const C<R> *pb = tile + (tid ^ xl) + (hb << 8);
        uint32_t jp[NW];
#pragma unroll
        for (int w = 0; w < NW; ++w) jp[w] = jpar[w] >> hb;
#pragma unroll
        for (int m = 0; m < PER / 2; ++m) step(widen<R>(po[m << 9]), widen<R>(pb[m << 9]), 2 * m, jp, m & 1);
    }
    const int lane = tid & 31;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        if (w >= nw) break;
        const double s = warp_sum(sg[w] * (acc[0][w] + acc[1][w]));  // sg holds the thread's Z parity
        if (lane == 0) s_acc_warp[w0 + w] += s;
    }
}
template <typename R, int NW, int KIND>
__device__ __forceinline__ void tiled_run_tb(int tb, const C<R> *tile, const C<R> (&v)[PTile<R>::per], int tid,
                                             uint32_t xl, int w0, int nw, const uint32_t *s_word,
                                             const uint32_t *s_jpar, uint32_t tmask, double *acc) {
    switch (tb) {
    case 0: tiled_run<R, NW, KIND, 0>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc); break;
    case 1: tiled_run<R, NW, KIND, 1>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc); break;
    case 2: tiled_run<R, NW, KIND, 2>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc); break;
    case 3: tiled_run<R, NW, KIND, 3>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc); break;
    case 4:
        if constexpr (PTile<R>::rbits > 4) tiled_run<R, NW, KIND, 4>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc);
        break;
    default: tiled_run<R, NW, KIND, -1>(tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc); break;
    }
}
template <typename R>
__global__ void __launch_bounds__(kPTileThreads, 2) k_pauli_tiled(const C<R> *__restrict__ a, PauliTiledP p,
                                                                  double *partials) {
    constexpr int TILE = PTile<R>::bits, PER = PTile<R>::per;
    extern __shared__ __align__(16) unsigned char pt_raw[];
    C<R> *tile = reinterpret_cast<C<R> *>(pt_raw);
    __shared__ uint8_t s_lbits[kPTileMaxBits], s_gbits[52];
    __shared__ uint64_t s_hi[PER];
    __shared__ double s_acc[kPTileThreads / 32][kPTileMaxWords];
    __shared__ uint32_t s_word[kPTileMaxWords], s_jpar[kPTileMaxWords], s_run[kPTileMaxWords];
    __shared__ uint32_t s_tmask;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid < TILE) s_lbits[tid] = p.lbits[tid];
    if (tid < 52) s_gbits[tid] = p.gbits[tid];
    if (tid < p.nterms) {
        s_word[tid] = tiled_word_bits(p.zl[tid], p.ny[tid]);
        s_jpar[tid] = tiled_reg_parity(p.zl[tid]);
    }
    if (tid < p.nruns)
        s_run[tid] = p.xl[tid] | ((uint32_t)p.run_begin[tid] << 13) |
                     ((uint32_t)(p.run_begin[tid + 1] - p.run_begin[tid]) << 19) | ((uint32_t)p.run_kinds[tid] << 22);
    static_assert(kPTileThreads == (kPTileThreads / 32) * kPTileMaxWords, "one accumulator per thread");
    (&s_acc[0][0])[tid] = 0.0;
    __syncthreads();
    if (tid < PER) s_hi[tid] = deposit_bits_u8((uint64_t)tid * kPTileThreads, s_lbits, TILE);
    __syncthreads();
    const uint64_t lo = deposit_bits_u8(tid, s_lbits, 8);
    const uint64_t zg = lane < p.nterms ? p.zg[lane] : 0;
    for (uint64_t tt = blockIdx.x; tt < p.ntiles; tt += gridDim.x) {
        const uint64_t tbase = deposit_bits_u8(tt, s_gbits, p.ng);
        C<R> v[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) v[j] = a[tbase | lo | s_hi[j]];
        __syncthreads();  // the previous tile has been read
#pragma unroll
        for (int j = 0; j < PER; ++j) tile[tid + j * kPTileThreads] = v[j];
        if (warp == 0) {  // parity of each word's Z factors outside the tile, one bit per word
            const uint32_t m = __ballot_sync(0xffffffffu, __popcll(tbase & zg) & 1);
            if (lane == 0) s_tmask = m;
        }
        __syncthreads();
        const uint32_t tmask = s_tmask;
        for (int run = 0; run < p.nruns; ++run) {
            const uint32_t rd = s_run[run];
            const uint32_t xl = rd & 0x1fffu;
            const int w0 = (rd >> 13) & 63, nw = (rd >> 19) & 7, kinds = (rd >> 22) & 3;
            const uint32_t xj = xl >> 8;
            const int tb = xj ? 31 - __clz(xj) : -1;
            double *acc = s_acc[warp];
            if (nw == 1) {
                if (kinds == 2) tiled_run_tb<R, 1, 1>(tb, tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc);
                else tiled_run_tb<R, 1, 0>(tb, tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc);
            } else if (nw == 2) {
                tiled_run_tb<R, 2, 2>(tb, tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc);
            } else {
                tiled_run_tb<R, 4, 2>(tb, tile, v, tid, xl, w0, nw, s_word, s_jpar, tmask, acc);
            }
        }
    }
    __syncthreads();
    if (tid < p.nterms) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kPTileThreads / 32; ++w) s += s_acc[w][tid];
        partials[(size_t)tid * gridDim.x + blockIdx.x] = s;
    }
}

uint64_t pauli_tile_bits(uint64_t xunion, uint32_t nq, size_t amp_bytes) {
    const int low = kPTileLowBits[amp_bytes == 16 ? 1 : 0];
    const int tbits = amp_bytes == 16 ? PTile<double>::bits : PTile<float>::bits;
    uint64_t in = xunion | ((uint64_t(1) << std::min<uint32_t>(low, nq)) - 1);
    if (nq < (uint32_t)tbits || __builtin_popcountll(in) > tbits) return 0;
    for (uint32_t b = 0; b < nq && __builtin_popcountll(in) < tbits; ++b) in |= uint64_t(1) << b;
    return in;
}

template <typename R>
void reduce_pauli_tiled(const void *psi, uint32_t nq, const PauliWord *terms, int nterms, double *partials,
                        double *out, cudaStream_t st) {
    if (nterms <= 0) return;
    if (nterms > kPTileMaxWords) throw ArgError("at most 32 Pauli words per tiled pass");
    uint64_t xu = 0;
    for (int t = 0; t < nterms; ++t) {
        if (!terms[t].xmask) throw ArgError("tiled Pauli pass takes words with X factors");
        if (t && terms[t].xmask < terms[t - 1].xmask) throw ArgError("tiled Pauli pass takes words sorted by X mask");
        xu |= terms[t].xmask;
    }
    const uint64_t in = pauli_tile_bits(xu, nq, sizeof(C<R>));
    if (!in) throw ArgError("Pauli X masks do not fit one tile");
    PauliTiledP p{};
    int loc[64];
    int nl = 0, ng = 0;
    for (uint32_t b = 0; b < nq; ++b) {
        loc[b] = -1;
        if ((in >> b) & 1) {
            loc[b] = nl;
            p.lbits[nl++] = (uint8_t)b;
        } else {
            p.gbits[ng++] = (uint8_t)b;
        }
    }
    p.ng = ng;
    p.ntiles = uint64_t(1) << (nq - PTile<R>::bits);
    p.nterms = nterms;
    auto local = [&](uint64_t m) {
        uint32_t r = 0;
        for (uint32_t b = 0; b < nq; ++b)
            if (((m >> b) & 1) && loc[b] >= 0) r |= 1u << loc[b];
        return r;
    };
    int nr = 0;
    for (int t = 0; t < nterms; ++t) {
        if (t == 0 || terms[t].xmask != terms[t - 1].xmask || t - p.run_begin[nr - 1] == 4) {
            p.run_begin[nr] = (uint8_t)t;
            p.xl[nr++] = local(terms[t].xmask);
        }
        p.zl[t] = local(terms[t].zmask);
        p.zg[t] = terms[t].zmask & ~in;
        p.ny[t] = (uint8_t)(terms[t].ny & 3);
        p.run_kinds[nr - 1] |= (p.ny[t] & 1) ? 2 : 1;
    }
    p.run_begin[nr] = (uint8_t)nterms;
    p.nruns = nr;
    const size_t smem = sizeof(C<R>) << PTile<R>::bits;
    const uint64_t nb = std::min<uint64_t>(p.ntiles, std::min<uint64_t>((uint64_t)sm_count() * 2, kMaxRedBlocks));
    B200SV_CUDA(cudaFuncSetAttribute(k_pauli_tiled<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_pauli_tiled<R><<<(unsigned)nb, kPTileThreads, smem, st>>>(static_cast<const C<R> *>(psi), p, partials);
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, (int)nb, nterms, out, 1, 1.0, st);
}

// ---- diagonal Pauli words (Z and I factors only), any number in one pass -----------------
// Per tile of 4096 consecutive amplitudes (state bits 0-11), the Walsh-Hadamard transform of
// the probabilities, W[k] = sum_m (-1)^popcount(m & k) p_(base + m), holds every diagonal
// word's restriction to the tile: <Z_z> gains (-1)^popcount(tile & (z >> 12)) W[z & 4095].
// The transform costs twelve FP64 additions per amplitude whatever the number of words: each
// thread holds 16 values and transforms four bits in registers, three times, with the tile
// passed through shared memory between (bits 8-11, then 4-7, then 0-3; the stages commute),
// under an XOR swizzle that keeps every phase's accesses free of bank conflicts.  Thread t
// then accumulates word t.  256 threads.
constexpr int kDiagThreads = 256;
constexpr int kDiagMaxWords = 256;
constexpr int kDiagTileBits = 12;
struct PauliDiagP {
    uint64_t ntiles;
    int nwords;
};
__device__ __forceinline__ int diag_pos(int m) { return m ^ ((m >> 4) & 15); }
__device__ __forceinline__ void fwht16(double (&v)[16]) {
#pragma unroll
    for (int h = 1; h < 16; h <<= 1) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            if (!(i & h)) {
                const double a = v[i], b = v[i + h];
                v[i] = a + b;
                v[i + h] = a - b;
            }
        }
    }
}
template <typename R>
__global__ void __launch_bounds__(kDiagThreads) k_pauli_diag(const C<R> *__restrict__ a, PauliDiagP p,
                                                             const uint64_t *__restrict__ zmask, double *partials) {
    __shared__ double w[1 << kDiagTileBits];
    const int t = threadIdx.x;
    const bool has_word = t < p.nwords;
    const uint64_t z = has_word ? zmask[t] : 0;
    const int zlo = (int)(z & ((1u << kDiagTileBits) - 1));
    const uint64_t zhi = z >> kDiagTileBits;
    double acc = 0.0;
    for (uint64_t tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
        const C<R> *src = a + (tile << kDiagTileBits);
        double v[16];
        // bits 8-11 in registers: element m = t + 256 r (coalesced loads)
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const double2 x = widen<R>(src[t + 256 * r]);
            v[r] = x.x * x.x + x.y * x.y;
        }
        fwht16(v);
        __syncthreads();  // the previous tile's words have read w
#pragma unroll
        for (int r = 0; r < 16; ++r) w[diag_pos(t + 256 * r)] = v[r];
        __syncthreads();
        // bits 4-7: m = (t & 15) | r << 4 | (t >> 4) << 8
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = w[diag_pos((t & 15) | (r << 4) | ((t >> 4) << 8))];
        fwht16(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) w[diag_pos((t & 15) | (r << 4) | ((t >> 4) << 8))] = v[r];
        __syncthreads();
        // bits 0-3: m = r | t << 4
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = w[diag_pos(r | (t << 4))];
        fwht16(v);
#pragma unroll
        for (int r = 0; r < 16; ++r) w[diag_pos(r | (t << 4))] = v[r];
        __syncthreads();
        if (has_word) {
            const double x = w[diag_pos(zlo)];
            acc += (__popcll(tile & zhi) & 1) ? -x : x;
        }
    }
    if (has_word) partials[(size_t)t * gridDim.x + blockIdx.x] = acc;
}

template <typename R>
void reduce_pauli_diag(const void *psi, uint32_t nq, const uint64_t *zmask_dev, int nwords, double *partials,
                       size_t partials_cap, double *out, cudaStream_t st) {
    if (nwords <= 0) return;
    if (nwords > kDiagMaxWords) throw ArgError("at most 256 diagonal Pauli words per pass");
    if (nq < (uint32_t)kDiagTileBits) throw Unsupported("diagonal Pauli pass needs at least 12 qubits");
    PauliDiagP p{};
    p.ntiles = uint64_t(1) << (nq - kDiagTileBits);
    p.nwords = nwords;
    const uint64_t cap = std::min<uint64_t>(kMaxRedBlocks, partials_cap / (size_t)nwords);
    const int nb = (int)std::max<uint64_t>(1, std::min<uint64_t>(p.ntiles, cap));
    k_pauli_diag<R><<<nb, kDiagThreads, 0, st>>>(static_cast<const C<R> *>(psi), p, zmask_dev, partials);
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, nwords, out, 1, 1.0, st);
}

template <typename R>
void reduce_pauli_multi(const void *psi, uint32_t nq, const PauliWord *terms, int nterms, double *partials,
                        double *out, cudaStream_t st) {
    if (nterms <= 0) return;
    if (nterms > 32) throw ArgError("at most 32 Pauli words per pass");
    PauliMultiP p{};
    p.n = uint64_t(1) << nq;
    p.nterms = nterms;
    for (int t = 0; t < nterms; ++t) {
        p.xmask[t] = terms[t].xmask;
        p.zmask[t] = terms[t].zmask;
        const int ny = terms[t].ny & 3;  // Re(i^ny z): z.re, -z.im, -z.re, z.im
        p.cr[t] = ny == 0 ? 1.0 : ny == 2 ? -1.0 : 0.0;
        p.ci[t] = ny == 1 ? -1.0 : ny == 3 ? 1.0 : 0.0;
        p.newx[t] = (t == 0 || terms[t].xmask != terms[t - 1].xmask) ? 1 : 0;
    }
    const int nb = red_blocks(p.n);
    const C<R> *a = static_cast<const C<R> *>(psi);
    if (nq <= 32) {
        if (nterms <= 8) k_pauli_multi<R, 8, uint32_t><<<nb, kRT, 0, st>>>(a, p, partials);
        else k_pauli_multi<R, 32, uint32_t><<<nb, kRT, 0, st>>>(a, p, partials);
    } else {
        if (nterms <= 8) k_pauli_multi<R, 8, uint64_t><<<nb, kRT, 0, st>>>(a, p, partials);
        else k_pauli_multi<R, 32, uint64_t><<<nb, kRT, 0, st>>>(a, p, partials);
    }
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, nterms, out, 1, 1.0, st);
}


template <typename R>
void reduce_dense_expval(const void *psi, uint32_t nq, const GateDesc &g, void *dev_matrix, double *partials,
                         double *out, cudaStream_t st) {
    if (g.kind != Kind::Dense || g.k > 4 || !g.cbits.empty()) throw Unsupported("dense expval needs k <= 4");
    DenseEvP<R> p{};
    p.ins = insert_of(g.tbits);
    p.k = g.k;
    p.ngroups = uint64_t(1) << (nq - g.k);
    for (int r = 0; r < (1 << g.k); ++r) {
        uint64_t o = 0;
        for (int j = 0; j < g.k; ++j)
            if (r & (1 << (g.k - 1 - j))) o |= uint64_t(1) << g.tbits[j];
        p.off[r] = o;
    }
    std::vector<C<R>> hm(g.m.size());
    for (size_t i = 0; i < g.m.size(); ++i) hm[i] = cvt<R>(g.m[i]);
    B200SV_CUDA(cudaMemcpyAsync(dev_matrix, hm.data(), hm.size() * sizeof(C<R>),
                                cudaMemcpyHostToDevice, st));
    const int nb = red_blocks(p.ngroups);
    const C<R> *a = static_cast<const C<R> *>(psi), *m = static_cast<const C<R> *>(dev_matrix);
    switch (g.k) {
    case 1: k_dense_ev<R, 1><<<nb, kRT, 0, st>>>(a, p, m, partials); break;
    case 2: k_dense_ev<R, 2><<<nb, kRT, 0, st>>>(a, p, m, partials); break;
    case 3: k_dense_ev<R, 3><<<nb, kRT, 0, st>>>(a, p, m, partials); break;
    default: k_dense_ev<R, 4><<<nb, kRT, 0, st>>>(a, p, m, partials); break;
    }
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, 1, out, 1, 1.0, st);
}

template <typename R> GenP<R> make_genp(uint32_t nq, const GateDesc &g);

template <typename R>
void reduce_generator_inner_complex(const void *bra, const void *ket, uint32_t nq, const GateDesc &g,
                                    double *partials, double *out2, cudaStream_t st) {
    GenP<R> p = make_genp<R>(nq, g);
    const int nb = red_blocks(p.ngroups);
    with_gen_form<R>(p, GoGenC<R>{nb, st, static_cast<const C<R> *>(bra), static_cast<const C<R> *>(ket), p, partials});
    B200SV_CUDA(cudaGetLastError());
    finalize(partials, nb, 2, out2, 1, 1.0, st);
}

template <typename R> GenP<R> make_genp(uint32_t nq, const GateDesc &g) {
    GenP<R> p{};
    p.kind = (int)g.kind;
    p.k = g.k;
    if (!g.cbits.empty()) throw Unsupported("generator forms carry no control bits");
    if (g.kind == Kind::Parity) {
        p.ngroups = uint64_t(1) << nq;
        p.pmask = g.pmask;
        p.pph[0] = cvt<R>(g.pphase[0]);
        p.pph[1] = cvt<R>(g.pphase[1]);
    } else {
        if (g.k > 4 || (g.kind == Kind::Dense && g.k > 2) || (g.kind == Kind::Diag && g.k > 2))
            throw Unsupported("generator form too wide");
        p.ins = insert_of(g.tbits);
        p.ngroups = uint64_t(1) << (nq - g.k);
        for (int r = 0; r < (1 << g.k); ++r) {
            uint64_t o = 0;
            for (int j = 0; j < g.k; ++j)
                if (r & (1 << (g.k - 1 - j))) o |= uint64_t(1) << g.tbits[j];
            p.off[r] = o;
        }
        for (size_t i = 0; i < g.m.size() && i < 16; ++i) p.m[i] = cvt<R>(g.m[i]);
        for (int i = 0; i < 4; ++i) p.m2[i] = cvt<R>(g.m2[i]);
        p.gamma = cvt<R>(g.gamma);
        p.pa = (int)g.pa;
        p.pb = (int)g.pb;
    }
    return p;
}

template <typename R>
void reduce_generator_inner(void *const *bras, int nbra, const void *ket, uint32_t nq, const GateDesc &g,
                            double alpha, double *partials, double *out, int out_stride, cudaStream_t st,
                            unsigned int *arrival) {
    if (nbra <= 0) return;
    if (nbra > 16) throw ArgError("at most 16 bras per generator product");
    GenP<R> p = make_genp<R>(nq, g);
    Bras<R> B{};
    for (int o = 0; o < nbra; ++o) B.p[o] = static_cast<const C<R> *>(bras[o]);
    const int nb = red_blocks(p.ngroups);
    const C<R> *k = static_cast<const C<R> *>(ket);
    const GenFinal fin{arrival, out, out_stride, alpha};
    with_gen_form<R>(p, GoGen<R>{nb, nbra, st, B, k, p, partials, fin});
    B200SV_CUDA(cudaGetLastError());
    if (arrival == nullptr) finalize(partials, nb, nbra, out, out_stride, alpha, st);
}

// ---- one adjoint step of a one-wire rotation, fused -------------------------------------
// At a differentiated one-wire gate the sweep needs -2 scale Im<bra_o|G|lambda> for every
// bra and then U^dagger applied to lambda and to every bra.  Both act on the same amplitude
// pairs, so one pass reads each pair once: the products come from the pair's values before
// the update, then the pair is updated in place (CAcc, as the gate kernels).  The results
// are formed by the last block (GenFinal).
struct AdjRotP {
    uint64_t npairs, low;  // (1 << bit) - 1
    uint64_t bit;
    double2 g[4];          // generator, row-major
    int nbra;
};
template <typename R> struct AdjRotMat {
    C<R> u[4];  // the inverse gate, row-major
};
template <typename R> struct MutBras {
    C<R> *p[16];  // the bras, updated in place
};
template <typename R, int NB>
__global__ void __launch_bounds__(kRT) k_adj_rot(C<R> *__restrict__ lambda, MutBras<R> bras, AdjRotP p,
                                                 AdjRotMat<R> um, double *partials, GenFinal fin) {
    __shared__ double sm[NB * 32];
    double acc[NB];
#pragma unroll
    for (int o = 0; o < NB; ++o) acc[o] = 0.0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t lo = g & p.low;
        const uint64_t i0 = ((g ^ lo) << 1) | lo, i1 = i0 | p.bit;
        const C<R> l0 = lambda[i0], l1 = lambda[i1];
        const double2 a0 = widen<R>(l0), a1 = widen<R>(l1);
        // w = G (a0, a1)
        const double2 w0 = make_double2(p.g[0].x * a0.x - p.g[0].y * a0.y + p.g[1].x * a1.x - p.g[1].y * a1.y,
                                        p.g[0].x * a0.y + p.g[0].y * a0.x + p.g[1].x * a1.y + p.g[1].y * a1.x);
        const double2 w1 = make_double2(p.g[2].x * a0.x - p.g[2].y * a0.y + p.g[3].x * a1.x - p.g[3].y * a1.y,
                                        p.g[2].x * a0.y + p.g[2].y * a0.x + p.g[3].x * a1.y + p.g[3].y * a1.x);
#pragma unroll
        for (int o = 0; o < NB; ++o) {
            if (o < p.nbra) {
                C<R> *b = bras.p[o];
                const C<R> c0 = b[i0], c1 = b[i1];
                const double2 b0 = widen<R>(c0), b1 = widen<R>(c1);
                acc[o] += (b0.x * w0.y - b0.y * w0.x) + (b1.x * w1.y - b1.y * w1.x);  // Im conj(b) w
                CAcc<R> x, y;
                x.add(um.u[0], c0);
                x.add(um.u[1], c1);
                y.add(um.u[2], c0);
                y.add(um.u[3], c1);
                b[i0] = x.get();
                b[i1] = y.get();
            }
        }
        CAcc<R> x, y;
        x.add(um.u[0], l0);
        x.add(um.u[1], l1);
        y.add(um.u[2], l0);
        y.add(um.u[3], l1);
        lambda[i0] = x.get();
        lambda[i1] = y.get();
    }
    block_reduce<NB>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int o = 0; o < NB; ++o)
            if (o < p.nbra) partials[(size_t)o * gridDim.x + blockIdx.x] = acc[o];
    }
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(fin.count, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = warp; o < p.nbra; o += (int)(blockDim.x >> 5)) {
        double v = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) v += __ldcg(&partials[(size_t)o * gridDim.x + b]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) fin.out[(size_t)o * fin.stride] = fin.alpha * v;
    }
    if (threadIdx.x == 0) *fin.count = 0u;
}

template <typename R>
void adjoint_rot_step(void *lambda, void *const *bras, int nbra, uint32_t nq, uint32_t bit, const cd (&g)[4],
                      const cd (&u)[4], double alpha, double *partials, double *out, int out_stride,
                      unsigned int *arrival, cudaStream_t st) {
    if (nbra <= 0 || nbra > 16) throw ArgError("one-wire adjoint step takes 1..16 bras");
    AdjRotP p{};
    p.npairs = uint64_t(1) << (nq - 1);
    p.bit = uint64_t(1) << bit;
    p.low = p.bit - 1;
    for (int i = 0; i < 4; ++i) p.g[i] = make_double2(g[i].real(), g[i].imag());
    p.nbra = nbra;
    AdjRotMat<R> um{};
    for (int i = 0; i < 4; ++i) um.u[i] = cvt<R>(u[i]);
    MutBras<R> B{};
    for (int o = 0; o < nbra; ++o) B.p[o] = static_cast<C<R> *>(bras[o]);
    const int nb = red_blocks(p.npairs);
    const GenFinal fin{arrival, out, out_stride, alpha};
    C<R> *lam = static_cast<C<R> *>(lambda);
    if (nbra == 1) k_adj_rot<R, 1><<<nb, kRT, 0, st>>>(lam, B, p, um, partials, fin);
    else if (nbra <= 4) k_adj_rot<R, 4><<<nb, kRT, 0, st>>>(lam, B, p, um, partials, fin);
    else k_adj_rot<R, 16><<<nb, kRT, 0, st>>>(lam, B, p, um, partials, fin);
    B200SV_CUDA(cudaGetLastError());
}

template <typename R>
void reduce_probs(const void *psi, uint32_t nq, const std::vector<uint32_t> &bits, double *partials,
                  size_t partials_cap, double *out, cudaStream_t st) {
    const C<R> *a = static_cast<const C<R> *>(psi);
    const int k = (int)bits.size();
    const uint64_t n = uint64_t(1) << nq;
    bool identity = (k == (int)nq);
    for (int j = 0; identity && j < k; ++j) identity = (bits[j] == nq - 1 - (uint32_t)j);
    if (identity) {
        k_probs_all<R><<<ew_grid(n), kRT, 0, st>>>(a, n, out);
        B200SV_CUDA(cudaGetLastError());
        return;
    }
    ProbsP p{};
    p.others = insert_of(bits);
    p.k = k;
    p.nothers = uint64_t(1) << (nq - k);
    p.nbins = uint64_t(1) << k;
    for (int j = 0; j < k; ++j) p.binmask[j] = uint64_t(1) << bits[j];
    if (k <= 12) {
        const uint64_t rows = (p.nbins + 7) / 8;
        uint64_t nbx = std::max<uint64_t>(1, std::min<uint64_t>((p.nothers + kRT * 4 - 1) / (kRT * 4),
                                                                 std::max<uint64_t>(1, kMaxRedBlocks / rows)));
        while (nbx > 1 && nbx * p.nbins > partials_cap) nbx /= 2;
        k_probs_hist<R><<<dim3((unsigned)nbx, (unsigned)rows), kRT, 0, st>>>(a, p, partials);
        B200SV_CUDA(cudaGetLastError());
        k_finalize<<<(unsigned)p.nbins, 128, 0, st>>>(partials, (int)nbx, out, 1, 1.0);
        B200SV_CUDA(cudaGetLastError());
    } else {
        k_probs_perbin<R><<<ew_grid(p.nbins), kRT, 0, st>>>(a, p, out);
        B200SV_CUDA(cudaGetLastError());
    }
}

template <typename R> void set_basis(void *psi, uint32_t nq, uint64_t index, cudaStream_t st) {
    B200SV_CUDA(cudaMemsetAsync(psi, 0, sizeof(C<R>) << nq, st));
    k_set_one<R><<<1, 1, 0, st>>>(static_cast<C<R> *>(psi), index);
    B200SV_CUDA(cudaGetLastError());
}

template <typename R>
void axpy_pauli(void *acc, const void *psi, uint32_t nq, const PauliWord &w, double c, cudaStream_t st) {
    const uint64_t n = uint64_t(1) << nq;
    k_axpy_pauli<R><<<ew_grid(n), kRT, 0, st>>>(static_cast<C<R> *>(acc), static_cast<const C<R> *>(psi), n,
                                                w.xmask, w.zmask, w.ny, c);
    B200SV_CUDA(cudaGetLastError());
}

template <typename R> void axpy(void *acc, const void *x, uint32_t nq, double c, cudaStream_t st) {
    const uint64_t n = uint64_t(1) << nq;
    k_axpy<R><<<ew_grid(n), kRT, 0, st>>>(static_cast<C<R> *>(acc), static_cast<const C<R> *>(x), n, c);
    B200SV_CUDA(cudaGetLastError());
}

#define B200SV_INST(R)                                                                                          \
    template void reduce_norm2<R>(const void *, uint32_t, double *, double *, cudaStream_t);                    \
    template void reduce_inner<R>(const void *, const void *, uint32_t, double *, double *, cudaStream_t);      \
    template void reduce_pauli_group<R>(const void *, uint32_t, const PauliWord *, int, double *, double *,     \
                                        cudaStream_t, bool);                                                    \
    template void reduce_pauli_diag<R>(const void *, uint32_t, const uint64_t *, int, double *, size_t,         \
                                       double *, cudaStream_t);                                                 \
    template void reduce_pauli_multi<R>(const void *, uint32_t, const PauliWord *, int, double *, double *,     \
                                        cudaStream_t);                                                          \
    template void reduce_dense_expval<R>(const void *, uint32_t, const GateDesc &, void *, double *,      \
                                         double *, cudaStream_t);                                               \
    template void reduce_generator_inner<R>(void *const *, int, const void *, uint32_t, const GateDesc &,       \
                                            double, double *, double *, int, cudaStream_t, unsigned int *);     \
    template void reduce_generator_inner_complex<R>(const void *, const void *, uint32_t, const GateDesc &,     \
                                                    double *, double *, cudaStream_t);                          \
    template void reduce_pauli_tiled<R>(const void *, uint32_t, const PauliWord *, int, double *, double *,     \
                                        cudaStream_t);                                                          \
    template void adjoint_rot_step<R>(void *, void *const *, int, uint32_t, uint32_t, const cd(&)[4],          \
                                      const cd(&)[4], double, double *, double *, int, unsigned int *,         \
                                      cudaStream_t);                                                           \
    template void reduce_probs<R>(const void *, uint32_t, const std::vector<uint32_t> &, double *, size_t,      \
                                  double *, cudaStream_t);                                                      \
    template void set_basis<R>(void *, uint32_t, uint64_t, cudaStream_t);                                       \
    template void axpy_pauli<R>(void *, const void *, uint32_t, const PauliWord &, double, cudaStream_t);       \
    template void axpy<R>(void *, const void *, uint32_t, double, cudaStream_t);
B200SV_INST(float)
B200SV_INST(double)

}  // namespace b200sv
