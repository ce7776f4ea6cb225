// sv_mcmc.cu — Metropolis-Hastings sampling of basis states.
//
// The reference runs one chain on the host (generate_samples_metropolis,
// LQ/measurements/MeasurementsLQubit.hpp:387-434; metropolis_step :612-640; proposals
// LQ/measurements/TransitionKernels.hpp:56-160): start at index 0, `num_burnin` steps,
// then one sample per step.  A step proposes t from the current index i and accepts
// it when U < min(1, |psi_t|^2 / |psi_i|^2).  Proposals:
//   local     — pick a bit position uniformly and a value 0/1 uniformly; the
//               proposal sets that bit to the value (no move when it already has it);
//   non-zero  — a basis index uniformly among those with |psi| > machine epsilon of
//               the state's precision.
// Here nchains independent chains run as GPU threads, each exactly that loop:
// chain c burns in, then gives samples c, c + nchains, c + 2 nchains, ... from its
// consecutive steps (nchains = 1 is the reference's single chain).  Every random
// number comes from Philox4x32-10 with counter (step_lo, step_hi, chain, 0x4D434D43)
// and key (seed_lo, seed_hi), so the samples are a deterministic function of the
// state, the seed and the chain count.  The acceptance test is evaluated as
// p_i == 0 or U * p_i < p_t with p = re*re + im*im in FP64 (no contraction), which
// equals U < min(1, p_t / p_i) without a logarithm or exponential.
// For non-zero proposals the candidates are found once per call: a bit per amplitude,
// per-256-amplitude counts and their exclusive prefix sums; a proposal draws
// r < total and locates the r-th candidate by a binary search over the prefixes and
// a scan of eight 32-bit words.
#include <algorithm>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr uint32_t kTag = 0x4D434D43u;
constexpr int kGroup = 256;  // amplitudes per candidate count (8 words of 32 bits)

struct P4 {
    uint32_t x0, x1, x2, x3;
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011).
__device__ __forceinline__ P4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed) {
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
    }
    return P4{c0, c1, c2, c3};
}

template <typename R> __device__ __forceinline__ double prob(const C<R> *psi, uint64_t i) {
    const double2 z = widen<R>(psi[i]);
    return __dadd_rn(__dmul_rn(z.x, z.x), __dmul_rn(z.y, z.y));
}

// candidate bits: word w holds amplitudes 32w .. 32w+31 (bit j = amplitude 32w+j)
template <typename R>
__global__ void k_nz_words(const C<R> *__restrict__ psi, uint64_t n, double thr, uint32_t *__restrict__ words,
                           uint64_t nwords) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t m = 0;
        for (int j = 0; j < 32; ++j) {
            const uint64_t i = w * 32 + j;
            if (i < n && prob<R>(psi, i) > thr) m |= 1u << j;
        }
        words[w] = m;
    }
}

__global__ void k_group_counts(const uint32_t *__restrict__ words, uint64_t nwords, uint64_t *__restrict__ counts,
                               uint64_t ngroups) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < ngroups; g += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0;
        for (int j = 0; j < kGroup / 32; ++j) {
            const uint64_t w = g * (kGroup / 32) + j;
            if (w < nwords) s += __popc(words[w]);
        }
        counts[g] = s;
    }
}

// Exclusive prefix sums of 1024-element blocks (256 threads x 4); block totals to `sums`.
// (in and out may be the same array: each thread reads its four values before writing them)
__global__ void __launch_bounds__(256) k_scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *sums) {
    __shared__ uint64_t wt[8];
    const uint64_t base = blockIdx.x * 1024ull + threadIdx.x * 4ull;
    uint64_t v[4], t = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        v[j] = base + j < n ? in[base + j] : 0;
        t += v[j];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t inc = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wt[warp] = inc;
    __syncthreads();
    uint64_t woff = 0;
    for (int w = 0; w < warp; ++w) woff += wt[w];
    uint64_t run = woff + inc - t;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (base + j < n) out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == 255) sums[blockIdx.x] = woff + inc;
}

__global__ void k_add_blocks(uint64_t *__restrict__ out, uint64_t n, const uint64_t *__restrict__ offs) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] += offs[i / 1024];
}

__global__ void k_total(const uint64_t *prefix, const uint64_t *counts, uint64_t ngroups, uint64_t *total) {
    *total = prefix[ngroups - 1] + counts[ngroups - 1];
}

unsigned ew_blocks(uint64_t n, int threads) {
    const uint64_t cap = uint64_t(sm_count()) * 16;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + threads - 1) / threads, cap));
}

// exclusive scan of n values; work holds the block sums of every level
void scan_u64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *work, cudaStream_t st) {
    const uint64_t nb = (n + 1023) / 1024;
    k_scan_u64<<<(unsigned)nb, 256, 0, st>>>(in, out, n, work);
    B200SV_CUDA(cudaGetLastError());
    if (nb > 1) {
        scan_u64(work, work, nb, work + nb, st);
        k_add_blocks<<<ew_blocks(n, 256), 256, 0, st>>>(out, n, work);
        B200SV_CUDA(cudaGetLastError());
    }
}

uint64_t scan_work(uint64_t n) {
    uint64_t w = 0;
    while (n > 1) {
        n = (n + 1023) / 1024;
        w += n;
    }
    return w + 1;
}

struct NzIndex {
    const uint32_t *words;
    const uint64_t *prefix;
    uint64_t ngroups, nwords;
    const uint64_t *total;
};

// the r-th candidate (r < total)
__device__ __forceinline__ uint64_t nz_pick(const NzIndex &z, uint64_t r) {
    uint64_t lo = 0, hi = z.ngroups;  // largest g with prefix[g] <= r
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (z.prefix[mid] <= r) lo = mid;
        else hi = mid;
    }
    uint64_t rem = r - z.prefix[lo];
    for (int j = 0; j < kGroup / 32 && lo * (kGroup / 32) + j < z.nwords; ++j) {
        uint32_t w = z.words[lo * (kGroup / 32) + j];
        const uint32_t pc = __popc(w);
        if (rem < pc) {
            for (uint64_t k = 0; k < rem; ++k) w &= w - 1;
            return lo * kGroup + j * 32 + (__ffs(w) - 1);
        }
        rem -= pc;
    }
    return lo * kGroup;  // not reached when r < total
}

template <typename R, int PROPOSAL>
__global__ void k_mcmc(const C<R> *__restrict__ psi, uint32_t nq, uint64_t burnin, uint64_t nshots, uint64_t nchains,
                       uint64_t seed, NzIndex z, uint64_t *__restrict__ out) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < nchains && c < nshots;
         c += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t nsamp = (nshots - c + nchains - 1) / nchains;
        const uint64_t total = PROPOSAL == B200SV_MCMC_NONZERO ? *z.total : 0;
        uint64_t idx = 0;
        double pi = prob<R>(psi, 0);
        for (uint64_t t = 0; t < burnin + nsamp; ++t) {
            const P4 x = philox((uint32_t)t, (uint32_t)(t >> 32), (uint32_t)c, kTag, seed);
            uint64_t trans;
            if (PROPOSAL == B200SV_MCMC_LOCAL) {
                const uint32_t site = (uint32_t)(((uint64_t)x.x0 * nq) >> 32);
                const uint64_t bit = uint64_t(1) << site;
                const uint64_t want = x.x1 & 1u;
                trans = (((idx >> site) & 1u) == want) ? idx : (idx ^ bit);
            } else {
                const uint64_t r64 = ((uint64_t)x.x1 << 32) | x.x0;
                trans = nz_pick(z, __umul64hi(r64, total));
            }
            const double pt = trans == idx ? pi : prob<R>(psi, trans);
            const double u = (double)((((uint64_t)x.x3 << 32) | x.x2) >> 11) * (1.0 / 9007199254740992.0);
            if (pi == 0.0 || __dmul_rn(u, pi) < pt) {
                idx = trans;
                pi = pt;
            }
            if (t >= burnin) out[c + (t - burnin) * nchains] = idx;
        }
    }
}

template <typename R>
void run_mcmc(const void *state, uint32_t nq, int proposal, uint64_t burnin, uint64_t nshots, uint64_t nchains,
              uint64_t seed, uint64_t *idx_dev, cudaStream_t st) {
    const uint64_t N = uint64_t(1) << nq;
    const C<R> *psi = static_cast<const C<R> *>(state);
    NzIndex z{};
    void *mem = nullptr;
    struct Free {
        void *&m;
        cudaStream_t s;
        ~Free() {
            if (m) cudaFreeAsync(m, s);
        }
    } fr{mem, st};
    if (proposal == B200SV_MCMC_NONZERO) {
        const uint64_t nwords = (N + 31) / 32, ngroups = (N + kGroup - 1) / kGroup;
        const uint64_t sw = scan_work(ngroups);
        const size_t bytes = nwords * 4 + (2 * ngroups + sw + 1) * 8 + 16;
        B200SV_CUDA(cudaMallocAsync(&mem, bytes, st));
        uint64_t *counts = reinterpret_cast<uint64_t *>(mem);
        uint64_t *prefix = counts + ngroups;
        uint64_t *work = prefix + ngroups;
        uint64_t *total = work + sw;
        uint32_t *words = reinterpret_cast<uint32_t *>(total + 1);
        const double eps = sizeof(R) == 4 ? 1.1920928955078125e-07 : 2.220446049250313e-16;  // 2^-23, 2^-52
        k_nz_words<R><<<ew_blocks(nwords, 256), 256, 0, st>>>(psi, N, eps * eps, words, nwords);
        B200SV_CUDA(cudaGetLastError());
        k_group_counts<<<ew_blocks(ngroups, 256), 256, 0, st>>>(words, nwords, counts, ngroups);
        B200SV_CUDA(cudaGetLastError());
        scan_u64(counts, prefix, ngroups, work, st);
        k_total<<<1, 1, 0, st>>>(prefix, counts, ngroups, total);
        B200SV_CUDA(cudaGetLastError());
        uint64_t h_total = 0;
        B200SV_CUDA(cudaMemcpyAsync(&h_total, total, 8, cudaMemcpyDeviceToHost, st));
        B200SV_CUDA(cudaStreamSynchronize(st));
        if (h_total == 0) throw ArgError("no basis state has a non-zero amplitude");
        z = NzIndex{words, prefix, ngroups, nwords, total};
    }
    const uint64_t active = std::min(nchains, nshots);
    const unsigned blocks = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((active + 127) / 128, uint64_t(1) << 20));
    if (proposal == B200SV_MCMC_LOCAL)
        k_mcmc<R, B200SV_MCMC_LOCAL><<<blocks, 128, 0, st>>>(psi, nq, burnin, nshots, nchains, seed, z, idx_dev);
    else
        k_mcmc<R, B200SV_MCMC_NONZERO><<<blocks, 128, 0, st>>>(psi, nq, burnin, nshots, nchains, seed, z, idx_dev);
    B200SV_CUDA(cudaGetLastError());
}

}  // namespace

void sample_mcmc(const void *state, uint32_t nq, int dtype, int proposal, uint64_t burnin, uint64_t nshots,
                 uint64_t nchains, uint64_t seed, uint64_t *idx_dev, cudaStream_t st) {
    if (proposal != B200SV_MCMC_LOCAL && proposal != B200SV_MCMC_NONZERO) throw ArgError("unknown MCMC proposal");
    if (nchains == 0) throw ArgError("the number of chains must be positive");
    if (nshots == 0) return;
    if (dtype == B200SV_C64) run_mcmc<float>(state, nq, proposal, burnin, nshots, nchains, seed, idx_dev, st);
    else run_mcmc<double>(state, nq, proposal, burnin, nshots, nchains, seed, idx_dev, st);
}

}  // namespace b200sv
