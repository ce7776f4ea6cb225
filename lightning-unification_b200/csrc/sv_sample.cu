// sv_sample.cu — inverse-CDF sampling with a reproducible CDF.
//
// Rule (lightning.kokkos, LK/measurements/MeasurementsKokkos.hpp:700-743 and
// LK/measurements/MeasuresFunctors.hpp:70-103): exclusive prefix sum of the
// probabilities, then per shot with uniform U: index 0 if U <= cdf[1], otherwise
// a binary search over (1, N] for the last cdf entry below U (cdf[N] taken as 1).
//
// The CDF association order is fixed so a CPU restatement can reproduce every
// bit of it:
//   p_i   = re*re + im*im in FP64, no contraction (complex64 widened first);
//   x_0   = p; level l groups x_l in runs of 32; E_l = sequential exclusive
//           prefix inside each run; x_{l+1}[g] = sequential sum of run g;
//   levels stop when one run covers the level; O_top = E_top;
//   O_l[j] = O_{l+1}[j / 32] + E_l[j]  (top down);  cdf = O_0.
//
// Only the run offsets O_1 (N / 32 doubles) are stored.  The search forms
// cdf[j] = O_1[j / 32] + (sequential sum of p over the first j mod 32 entries of
// run j / 32) when it needs it, with the same additions in the same order as the
// full CDF, so every compared value is bit-identical to it.  Searches that start
// at (1, N] probe indices of the form k * 2^m + 1 while the range is wide, so most
// probes add one probability; the state is read in place and no N-entry array is
// allocated (a 33-qubit complex64 state needs 2 GiB of offsets instead of a 64 GiB CDF).
// Each thread searches four shots in lock step, so four independent memory reads
// are in flight per thread.
#include <vector>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr int kRun = 32;      // elements per run (sequential inside)
constexpr int kST = 128;      // threads per block = runs per block
constexpr int kPad = kRun + 1;

template <typename R> __device__ __forceinline__ double prob_of(C<R> a) {
    const double re = (double)a.x, im = (double)a.y;
    return __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
}

// x1[g] = sequential sum of p over run g (level 0 from the state)
template <typename R>
__global__ void __launch_bounds__(kST) k_l0_totals(const C<R> *__restrict__ a, uint64_t n, double *__restrict__ x1) {
    __shared__ double s[kST * kPad];
    const uint64_t e0 = (uint64_t)blockIdx.x * kST * kRun;
    for (int e = threadIdx.x; e < kST * kRun; e += kST) {
        const uint64_t i = e0 + e;
        s[(e / kRun) * kPad + (e % kRun)] = i < n ? prob_of<R>(a[i]) : 0.0;
    }
    __syncthreads();
    const uint64_t g = (uint64_t)blockIdx.x * kST + threadIdx.x;
    const uint64_t nruns = (n + kRun - 1) / kRun;
    if (g < nruns) {
        const int cnt = (int)min((uint64_t)kRun, n - g * kRun);
        double acc = 0.0;
        for (int j = 0; j < cnt; ++j) acc = __dadd_rn(acc, s[threadIdx.x * kPad + j]);
        x1[g] = acc;
    }
}

// E (in place over x) = run-wise sequential exclusive prefix; xnext[g] = run total
__global__ void __launch_bounds__(kST) k_scan_level(double *__restrict__ x, uint64_t len, double *__restrict__ xnext) {
    __shared__ double s[kST * kPad];
    const uint64_t e0 = (uint64_t)blockIdx.x * kST * kRun;
    for (int e = threadIdx.x; e < kST * kRun; e += kST) {
        const uint64_t i = e0 + e;
        s[(e / kRun) * kPad + (e % kRun)] = i < len ? x[i] : 0.0;
    }
    __syncthreads();
    const uint64_t g = (uint64_t)blockIdx.x * kST + threadIdx.x;
    const uint64_t nruns = (len + kRun - 1) / kRun;
    if (g < nruns) {
        const int cnt = (int)min((uint64_t)kRun, len - g * kRun);
        double acc = 0.0;
        for (int j = 0; j < cnt; ++j) {
            const double v = s[threadIdx.x * kPad + j];
            s[threadIdx.x * kPad + j] = acc;
            acc = __dadd_rn(acc, v);
        }
        if (xnext) xnext[g] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kST * kRun; e += kST) {
        const uint64_t i = e0 + e;
        if (i < len) x[i] = s[(e / kRun) * kPad + (e % kRun)];
    }
}

// O_l[j] = O_{l+1}[j / 32] + E_l[j]
__global__ void k_add_offsets(const double *__restrict__ parent, double *__restrict__ e, uint64_t len) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < len; j += (uint64_t)gridDim.x * blockDim.x)
        e[j] = __dadd_rn(parent[j / kRun], e[j]);
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC 2011): counter = (i_lo, i_hi, 0, 0), key = (seed_lo, seed_hi);
// u = ((out1 << 32 | out0) >> 11) * 2^-53 in [0, 1).
__device__ __forceinline__ double philox_u01(uint64_t i, uint64_t seed) {
    uint32_t c0 = (uint32_t)i, c1 = (uint32_t)(i >> 32), c2 = 0, c3 = 0;
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
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    const uint64_t x = ((uint64_t)c1 << 32) | c0;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}
__global__ void k_philox(double *__restrict__ u, uint64_t n, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        u[i] = philox_u01(i, seed);
}

// cdf[j] of the rule (j < N): O_1[j / 32] plus the sequential sum of the run's first j mod 32
// probabilities, added in the order of the full CDF
template <typename R>
__device__ __forceinline__ double cdf_at(const C<R> *__restrict__ a, const double *__restrict__ o1, uint64_t j) {
    const uint64_t g = j >> 5;
    const int r = (int)(j & 31u);
    const double off = o1[g];
    double acc = 0.0;
    const C<R> *run = a + (g << 5);
    for (int i = 0; i < r; ++i) acc = __dadd_rn(acc, prob_of<R>(run[i]));
    return __dadd_rn(off, acc);
}

constexpr int kShotsPerThread = 4;

template <typename R>
__global__ void k_sample_runs(const C<R> *__restrict__ a, const double *__restrict__ o1, uint64_t N,
                              const double *__restrict__ u, uint64_t nshots, uint64_t *__restrict__ idx) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * kShotsPerThread;
    for (uint64_t k0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) * kShotsPerThread; k0 < nshots;
         k0 += stride) {
        double U[kShotsPerThread];
        uint64_t lo[kShotsPerThread], hi[kShotsPerThread];
        bool act[kShotsPerThread];
        const double c1 = N > 1 ? cdf_at<R>(a, o1, 1) : 1.0;
#pragma unroll
        for (int s = 0; s < kShotsPerThread; ++s) {
            const bool in = k0 + s < nshots;
            U[s] = in ? u[k0 + s] : 0.0;
            lo[s] = 1;
            hi[s] = N;
            // index 0 when U <= cdf[1]; the search runs for the others
            act[s] = in && !(U[s] <= c1);
            if (!act[s]) hi[s] = 1;
        }
        for (;;) {
            bool any = false;
#pragma unroll
            for (int s = 0; s < kShotsPerThread; ++s) {
                if (act[s] && hi[s] - lo[s] > 1) {
                    any = true;
                    const uint64_t mid = hi[s] - ((hi[s] - lo[s]) >> 1);
                    const double c = (mid == N) ? 1.0 : cdf_at<R>(a, o1, mid);
                    if (c < U[s]) lo[s] = mid;
                    else hi[s] = mid;
                }
            }
            if (!any) break;
        }
#pragma unroll
        for (int s = 0; s < kShotsPerThread; ++s)
            if (k0 + s < nshots) idx[k0 + s] = hi[s] - 1;
    }
}

std::vector<uint64_t> level_lengths(uint64_t n) {
    std::vector<uint64_t> L{n};
    while (L.back() > (uint64_t)kRun) L.push_back((L.back() + kRun - 1) / kRun);
    return L;  // L[0] = n; the last level fits in one run
}

dim3 ew(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    const uint64_t cap = uint64_t(sm_count()) * 16;
    return dim3((unsigned)std::max<uint64_t>(1, std::min(b, cap)));
}

}  // namespace

size_t run_offsets_doubles(uint64_t N) {
    auto L = level_lengths(N);
    size_t s = 1;
    for (size_t l = 1; l < L.size(); ++l) s += L[l];
    return s + (size_t)kRun;
}

template <typename R>
void build_run_offsets(const void *psi, uint32_t nq, double *work, cudaStream_t st) {
    const uint64_t n = uint64_t(1) << nq;
    const C<R> *a = static_cast<const C<R> *>(psi);
    const auto L = level_lengths(n);
    const uint64_t per_block = (uint64_t)kST * kRun;
    if (L.size() == 1) {  // one run: O_1 = [0]
        B200SV_CUDA(cudaMemsetAsync(work, 0, sizeof(double), st));
        return;
    }
    // x_l for l >= 1 live consecutively in work: x_1 at work + 0, x_2 after it, ...
    std::vector<double *> x(L.size());
    size_t off = 0;
    for (size_t l = 1; l < L.size(); ++l) {
        x[l] = work + off;
        off += L[l];
    }
    k_l0_totals<R><<<(unsigned)((n + per_block - 1) / per_block), kST, 0, st>>>(a, n, x[1]);
    B200SV_CUDA(cudaGetLastError());
    const size_t top = L.size() - 1;
    for (size_t l = 1; l <= top; ++l) {
        double *next = (l < top) ? x[l + 1] : nullptr;
        k_scan_level<<<(unsigned)((L[l] + per_block - 1) / per_block), kST, 0, st>>>(x[l], L[l], next);
        B200SV_CUDA(cudaGetLastError());
    }
    for (size_t l = top; l-- > 1;) {
        k_add_offsets<<<ew(L[l]), 256, 0, st>>>(x[l + 1], x[l], L[l]);
        B200SV_CUDA(cudaGetLastError());
    }
}

void philox_uniforms(double *u, uint64_t n, uint64_t seed, cudaStream_t st) {
    k_philox<<<ew(n), 256, 0, st>>>(u, n, seed);
    B200SV_CUDA(cudaGetLastError());
}

template <typename R>
void sample_runs(const void *psi, uint32_t nq, const double *o1, const double *u, uint64_t nshots, uint64_t *idx,
                 cudaStream_t st) {
    if (nshots == 0) return;
    k_sample_runs<R><<<ew((nshots + kShotsPerThread - 1) / kShotsPerThread), 256, 0, st>>>(
        static_cast<const C<R> *>(psi), o1, uint64_t(1) << nq, u, nshots, idx);
    B200SV_CUDA(cudaGetLastError());
}

template void build_run_offsets<float>(const void *, uint32_t, double *, cudaStream_t);
template void build_run_offsets<double>(const void *, uint32_t, double *, cudaStream_t);
template void sample_runs<float>(const void *, uint32_t, const double *, const double *, uint64_t, uint64_t *,
                                 cudaStream_t);
template void sample_runs<double>(const void *, uint32_t, const double *, const double *, uint64_t, uint64_t *,
                                  cudaStream_t);

}  // namespace b200sv
