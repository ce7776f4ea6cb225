// sv_gates.cu — gate application kernels (one HBM pass per gate).
//
// Every form walks the 2^(n-k-c) groups of a k-target, c-control gate with a
// grid-stride loop; consecutive threads take consecutive group indices, so the
// bits below the lowest gate bit map to consecutive addresses and each warp's
// loads coalesce into full 32-byte sectors.  complex128 amplitudes are loaded
// as one 128-bit double2, complex64 as a 64-bit float2.
//
// Replaces the per-gate loops of LQ/gates/cpu_kernels/GateImplementationsLM.hpp:204-1352
// and GateImplementationsPI.hpp:248-289 / :785-799 (same index mathematics,
// revWireParity generalised to any number of inserted bits).
#include <algorithm>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {

void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            throw AllocError(std::string("CUDA allocation failed: ") + what + ": " + cudaGetErrorString(e));
        }
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

int sm_count() {
    static std::mutex mu;
    static std::vector<int> cache;
    int dev = 0;
    B200SV_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
    if (cache[dev] == 0) {
        int n = 0;
        B200SV_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

namespace {

constexpr int kThreads = 256;

struct States {
    void *p[kMaxStatesPerLaunch];
};

Insert make_insert(std::vector<uint32_t> bits) {
    std::sort(bits.begin(), bits.end());
    Insert ins{};
    ins.nb = (int)bits.size();
    if (ins.nb > kMaxInsert) throw Unsupported("gate touches more than 16 bits");
    for (int j = 0; j < ins.nb; ++j) ins.low[j] = (uint64_t(1) << bits[j]) - 1;
    return ins;
}

// offsets of the 2^k rows of a group: row r has bit (k-1-j) set for target j
template <int MAXR>
void fill_offsets(uint64_t (&off)[MAXR], const std::vector<uint32_t> &tb) {
    const int k = (int)tb.size();
    for (int r = 0; r < (1 << k); ++r) {
        uint64_t o = 0;
        for (int j = 0; j < k; ++j)
            if (r & (1 << (k - 1 - j))) o |= uint64_t(1) << tb[j];
        off[r] = o;
    }
}

uint64_t ctrl_mask(const std::vector<uint32_t> &cb) {
    uint64_t m = 0;
    for (auto b : cb) m |= uint64_t(1) << b;
    return m;
}

// per_thread: work items a thread takes per trip (the kernels that batch their loads), so a
// small state gets one wave of threads that each keep several loads in flight
dim3 grid_for(uint64_t work, int nstates, int per_thread = 1) {
    const uint64_t cap = uint64_t(sm_count()) * 16;
    const uint64_t per_block = uint64_t(kThreads) * (uint64_t)per_thread;
    uint64_t b = (work + per_block - 1) / per_block;
    if (b > cap) b = cap;
    if (b == 0) b = 1;
    return dim3((unsigned)b, (unsigned)nstates);
}

// ---------------------------------------------------------------------------
template <typename R, int K> struct DenseP {
    Insert ins;
    uint64_t cmask, ngroups;
    uint64_t off[1 << K];
    C<R> m[(1 << K) * (1 << K)];
};
template <typename R, int K> struct DenseDevP {
    Insert ins;
    uint64_t cmask, ngroups;
    uint64_t off[1 << K];
    const C<R> *m;
};

template <typename R, int K>
__global__ void __launch_bounds__(kThreads) k_dense(States s, DenseP<R, K> p) {
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    constexpr int D = 1 << K;
    if constexpr (K == 1) {
        // one-wire steps: U pairs a trip, every load issued before the first store
        constexpr int U = 4;
        const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
        for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g0 < p.ngroups; g0 += U * stride) {
            uint64_t base[U];
            C<R> v0[U], v1[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint64_t g = g0 + u * stride;
                base[u] = g < p.ngroups ? (p.ins(g) | p.cmask) : ~uint64_t(0);
                if (g < p.ngroups) {
                    v0[u] = sv[base[u] + p.off[0]];
                    v1[u] = sv[base[u] + p.off[1]];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (base[u] == ~uint64_t(0)) continue;
                CAcc<R> a, b;
                a.set(p.m[0], v0[u]); a.add(p.m[1], v1[u]);
                b.set(p.m[2], v0[u]); b.add(p.m[3], v1[u]);
                sv[base[u] + p.off[0]] = a.get();
                sv[base[u] + p.off[1]] = b.get();
            }
        }
    } else {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g) | p.cmask;
        C<R> v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = sv[base + p.off[r]];
        if constexpr (K >= 3) {
            // two output rows per trip of a rolled loop: two accumulators live instead of
            // 2^K, so more warps fit on an SM (72 vs 108 registers for complex128 at K = 3,
            // which moves a 30-qubit 3-wire unitary from 4.5 to 6.1 TB/s); same FMA order.
            // At K = 4 (complex128, 30 qubits) this takes 9.2 ms; four rows a trip 9.8 ms,
            // every row unrolled 13.3 ms (172 registers)
#pragma unroll 1
            for (int r = 0; r < D; r += 2) {
                CAcc<R> a, b;
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    cacc_term<R>(a, c, p.m[r * D + c], v[c]);
                    cacc_term<R>(b, c, p.m[r * D + D + c], v[c]);
                }
                sv[base + p.off[r]] = a.get();
                sv[base + p.off[r + 1]] = b.get();
            }
        } else {
#pragma unroll
            for (int r = 0; r < D; ++r) {
                CAcc<R> a;
#pragma unroll
                for (int c = 0; c < D; ++c) cacc_term<R>(a, c, p.m[r * D + c], v[c]);
                sv[base + p.off[r]] = a.get();
            }
        }
    }
    }
}

// A one-wire matrix on state bit 0: the pair of a group is two adjacent amplitudes, which the
// group-per-thread kernel reads and writes with two half-used 32-byte sectors per access.
// Here each thread owns one amplitude (fully coalesced loads and stores), takes its partner
// from the neighbouring lane and forms its own output row with the same FMA order.
template <typename R> struct Dense1LowP {
    uint64_t n;
    C<R> m[4];
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_dense1_low(States s, Dense1LowP<R> p) {
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    // n and the stride are multiples of 32, so every lane of a warp makes the same trips
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < p.n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const C<R> v = sv[i];
        C<R> o;
        o.x = __shfl_xor_sync(0xffffffffu, v.x, 1);
        o.y = __shfl_xor_sync(0xffffffffu, v.y, 1);
        const bool hi = i & 1;
        CAcc<R> a;
        a.set(hi ? p.m[2] : p.m[0], hi ? o : v);
        a.add(hi ? p.m[3] : p.m[1], hi ? v : o);
        sv[i] = a.get();
    }
}

// A complex64 two-wire matrix on state bits 0 and 1 (no controls): a group's four amplitudes
// are 32 contiguous bytes, which the group-per-thread kernel reads with four 8-byte loads at a
// 32-byte stride across the warp.  Here each thread moves its group with two 16-byte loads and
// stores.  Matrix row r sits at memory slot r, or with rows 1 and 2 exchanged when the first
// target is bit 0 (SWAPMID); the sums run over the matrix columns in order, as in k_dense.
template <typename R> struct Dense2LowP {
    uint64_t ngroups;
    C<R> m[16];
};
template <bool SWAPMID>
__device__ __forceinline__ constexpr int slot2(int r) {
    return SWAPMID ? (r == 1 ? 2 : r == 2 ? 1 : r) : r;
}
template <bool SWAPMID>
__global__ void __launch_bounds__(kThreads) k_dense2_low(States s, Dense2LowP<float> p) {
    float4 *__restrict__ sv = static_cast<float4 *>(s.p[blockIdx.y]);
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const float4 lo = sv[2 * g], hi = sv[2 * g + 1];
        const float2 x[4] = {make_float2(lo.x, lo.y), make_float2(lo.z, lo.w), make_float2(hi.x, hi.y),
                             make_float2(hi.z, hi.w)};
        float2 y[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            CAcc<float> a;
#pragma unroll
            for (int c = 0; c < 4; ++c) cacc_term<float>(a, c, p.m[r * 4 + c], x[slot2<SWAPMID>(c)]);
            y[slot2<SWAPMID>(r)] = a.get();
        }
        sv[2 * g] = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
        sv[2 * g + 1] = make_float4(y[2].x, y[2].y, y[3].x, y[3].y);
    }
}

template <typename R, int K>
__global__ void __launch_bounds__(kThreads) k_dense_dev(States s, DenseDevP<R, K> p) {
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    constexpr int D = 1 << K;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g) | p.cmask;
        C<R> v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = sv[base + p.off[r]];
#pragma unroll 1
        for (int r = 0; r < D; r += 2) {
            CAcc<R> a, b;
#pragma unroll
            for (int c = 0; c < D; ++c) {
                cacc_term<R>(a, c, __ldg(&p.m[r * D + c]), v[c]);
                cacc_term<R>(b, c, __ldg(&p.m[r * D + D + c]), v[c]);
            }
            sv[base + p.off[r]] = a.get();
            sv[base + p.off[r + 1]] = b.get();
        }
    }
}

// Dense blocks on K = 5..10 target bits (compute-bound from K = 5 in FP64): a register-tiled
// complex matrix product.  Each CTA takes tiles of 4096 amplitudes — TG = 4096 / 2^K
// consecutive groups times all 2^K rows — staged in shared memory with coalesced loads
// (consecutive threads take consecutive groups), and each thread accumulates a 4 x 4 block
// of outputs: rows tr + i * RB and groups tg + j * TG / 4, so a warp's shared-memory reads
// are contiguous.  The matrix is passed transposed (mt[c * 2^K + r] = M[r][c]) and staged in
// chunks of CK columns (TiledShape); every output is the same ordered sum over c as in k_dense_dev, so
// results are bit-identical to it.  The outputs go back through the tile for coalesced
// stores, which also makes the in-place update safe (a tile's groups belong to one CTA).
constexpr int kTileAmps = 4096;
constexpr int kTiledThreads = 256;
template <int K> struct TiledShape {
    static constexpr int D = 1 << K;
    static constexpr int TG = kTileAmps / D;        // groups per tile
    static constexpr int RB = D / 4;                // row blocks
    // matrix columns per staged chunk: the whole matrix when 2^K <= 32, else two buffers of
    // 1024 entries, filled with cp.async one chunk ahead of the one being multiplied
    static constexpr bool kResident = D <= 32;
    static constexpr int CK = kResident ? D : 1024 / D;
    static constexpr int MSH = kResident ? D * D : 2 * 1024;  // staged matrix entries
    static_assert(kTiledThreads % TG == 0 && RB * (TG / 4) == kTiledThreads, "tile shape");
};
template <typename R, int K> struct TiledP {
    Insert ins;
    uint64_t cmask, ntiles;
    uint64_t off[1 << K];
    const C<R> *mt;
};
template <typename R, int K>
__global__ void __launch_bounds__(kTiledThreads, 2) k_dense_tiled(States s, TiledP<R, K> p) {
    using S = TiledShape<K>;
    constexpr int D = S::D, TG = S::TG, RB = S::RB, CK = S::CK, TG4 = TG / 4;
    constexpr bool kResident = S::kResident;
    constexpr int kPieces = CK * D * (int)sizeof(C<R>) / 16;  // 16-byte pieces per chunk
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C<R> *tile = reinterpret_cast<C<R> *>(smem_raw);
    C<R> *msh = tile + kTileAmps;
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    const int t = threadIdx.x;
    const int tr = t % RB, tg = t / RB;
    // Thread t moves tile elements e = t + 256 q: group e % TG = t % TG (TG divides 256) and
    // row t / TG + q * 256 / TG.  Tiles start at multiples of TG, so the bit insertion splits
    // into a per-tile part and this per-thread part (the two touch disjoint bits).
    constexpr int QS = kTiledThreads / TG;
    const uint64_t lo = p.ins((uint64_t)(t % TG));
    const int r0 = t / TG;
    if constexpr (kResident)
        for (int e = t; e < D * D; e += kTiledThreads) msh[e] = p.mt[e];
    auto stage = [&](int ci) {  // chunk ci (columns ci * CK ...) into buffer ci & 1
        const char *src = reinterpret_cast<const char *>(p.mt + (size_t)ci * CK * D);
        char *dst = reinterpret_cast<char *>(msh + (ci & 1) * CK * D);
        for (int e = t; e < kPieces; e += kTiledThreads) cp_async16(dst + 16 * e, src + 16 * e);
        cp_async_commit();
    };
    for (uint64_t ti = blockIdx.x; ti < p.ntiles; ti += gridDim.x) {
        const uint64_t base = p.ins(ti * TG) | p.cmask | lo;
        __syncthreads();  // the previous tile has been stored and its chunks read
        if constexpr (!kResident) stage(0);  // in flight during the tile load
#pragma unroll
        for (int q = 0; q < kTileAmps / kTiledThreads; ++q)
            tile[t + q * kTiledThreads] = sv[base + p.off[r0 + q * QS]];
        __syncthreads();
        CAcc<R> acc[4][4];
        for (int ci = 0; ci < D / CK; ++ci) {
            if constexpr (!kResident) {
                if (ci + 1 < D / CK) {
                    stage(ci + 1);
                    cp_async_wait1();  // chunk ci has landed (this thread's pieces)
                } else {
                    cp_async_wait0();
                }
                __syncthreads();  // ... and every thread's
            }
            const C<R> *mc = msh + (kResident ? 0 : (ci & 1) * CK * D);
            const C<R> *vc = tile + ci * CK * TG;
#pragma unroll 4
            for (int c = 0; c < CK; ++c) {
                C<R> m[4], v[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) m[i] = mc[c * D + tr + i * RB];
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = vc[c * TG + tg + j * TG4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j].add(m[i], v[j]);
            }
            if constexpr (!kResident) __syncthreads();  // buffer ci & 1 is refilled by stage(ci + 2)
        }
        __syncthreads();  // every thread has read the whole tile
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) tile[(tr + i * RB) * TG + tg + j * TG4] = acc[i][j].get();
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kTileAmps / kTiledThreads; ++q)
            sv[base + p.off[r0 + q * QS]] = tile[t + q * kTiledThreads];
    }
}

// Large dense blocks (k = 11, and 7..10 on states under 12 qubits): one CTA per group, the
// group staged in shared memory.
struct BigDenseP {
    Insert ins;
    uint64_t ngroups;
    uint64_t tmask[12];  // bit of target j (j = 0 is the matrix MSB)
    int k;
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_dense_big(States s, BigDenseP p, const C<R> *__restrict__ m) {
    extern __shared__ unsigned char smem_raw[];
    C<R> *vs = reinterpret_cast<C<R> *>(smem_raw);
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    const int D = 1 << p.k;
    for (uint64_t g = blockIdx.x; g < p.ngroups; g += gridDim.x) {
        const uint64_t base = p.ins(g);
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
            uint64_t o = 0;
            for (int j = 0; j < p.k; ++j)
                if (r & (1 << (p.k - 1 - j))) o |= p.tmask[j];
            vs[r] = sv[base + o];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < D; r += blockDim.x) {
            CAcc<R> a;
            const C<R> *row = m + (size_t)r * D;
            for (int c = 0; c < D; ++c) a.add(__ldg(&row[c]), vs[c]);
            uint64_t o = 0;
            for (int j = 0; j < p.k; ++j)
                if (r & (1 << (p.k - 1 - j))) o |= p.tmask[j];
            sv[base + o] = a.get();
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
template <typename R, int K> struct DiagP {
    Insert ins;
    uint64_t cmask, ngroups;
    uint64_t off[1 << K];
    C<R> ph[1 << K];
};
template <typename R, int K>
__global__ void __launch_bounds__(kThreads) k_diag(States s, DiagP<R, K> p) {
    // U groups a trip, every load issued before the first store (one multiply per amplitude
    // covers little of the load latency)
    constexpr int D = 1 << K, U = D >= 4 ? 2 : 4;
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g0 < p.ngroups; g0 += U * stride) {
        uint64_t base[U];
        C<R> v[U][D];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t g = g0 + u * stride;
            base[u] = g < p.ngroups ? (p.ins(g) | p.cmask) : ~uint64_t(0);
            if (g < p.ngroups) {
#pragma unroll
                for (int r = 0; r < D; ++r) v[u][r] = sv[base[u] + p.off[r]];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (base[u] == ~uint64_t(0)) continue;
#pragma unroll
            for (int r = 0; r < D; ++r) {
                CAcc<R> a;
                a.set(p.ph[r], v[u][r]);
                sv[base[u] + p.off[r]] = a.get();
            }
        }
    }
}

struct SwapP {
    Insert ins;
    uint64_t cmask, ngroups, oa, ob;
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_swap(States s, SwapP p) {
    // U groups a trip with every load issued before the first store: a swap has no arithmetic
    // to cover the load latency, so the loads in flight per thread set its bandwidth
    constexpr int U = 4;
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g0 < p.ngroups; g0 += U * stride) {
        uint64_t base[U];
        C<R> a[U], b[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t g = g0 + u * stride;
            base[u] = g < p.ngroups ? (p.ins(g) | p.cmask) : ~uint64_t(0);
            if (g < p.ngroups) {
                a[u] = sv[base[u] + p.oa];
                b[u] = sv[base[u] + p.ob];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (base[u] == ~uint64_t(0)) continue;
            sv[base[u] + p.oa] = b[u];
            sv[base[u] + p.ob] = a[u];
        }
    }
}

template <typename R, int K> struct PairP {
    Insert ins;
    uint64_t ngroups;
    uint64_t off[1 << K];
    int pa, pb, scale_rest;
    C<R> m2[4];
    C<R> gamma;
};
template <typename R, int K>
__global__ void __launch_bounds__(kThreads) k_pair(States s, PairP<R, K> p) {
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g);
        const C<R> va = sv[base + p.off[p.pa]];
        const C<R> vb = sv[base + p.off[p.pb]];
        CAcc<R> a, b;
        a.add(p.m2[0], va);
        a.add(p.m2[1], vb);
        b.add(p.m2[2], va);
        b.add(p.m2[3], vb);
        sv[base + p.off[p.pa]] = a.get();
        sv[base + p.off[p.pb]] = b.get();
        if (p.scale_rest) {
#pragma unroll
            for (int r = 0; r < (1 << K); ++r) {
                if (r == p.pa || r == p.pb) continue;
                const C<R> v = sv[base + p.off[r]];
                CAcc<R> c;
                c.add(p.gamma, v);
                sv[base + p.off[r]] = c.get();
            }
        }
    }
}

template <typename R> struct ParityP {
    uint64_t n, mask;
    C<R> ph[2];
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_parity(States s, ParityP<R> p) {
    // U amplitudes a trip, every load issued before the first store
    constexpr int U = 4;
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i0 < p.n; i0 += U * stride) {
        C<R> v[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (i0 + u * stride < p.n) v[u] = sv[i0 + u * stride];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t i = i0 + u * stride;
            if (i >= p.n) continue;
            CAcc<R> a;
            a.set((__popcll(i & p.mask) & 1) ? p.ph[1] : p.ph[0], v[u]);  // a select: an index would copy ph to local memory
            sv[i] = a.get();
        }
    }
}

template <typename R> C<R> cvt(const cd &z) { return mk<R>((R)z.real(), (R)z.imag()); }

// Returns false when no kernel of this family takes the gate (K = 7 on a state too small
// for one tile); the caller then uses k_dense_big.
template <typename R, int K>
bool launch_dense_k(const States &S, int ns, uint32_t nq, const GateDesc &g, void *scratch,
                    cudaStream_t st) {
    std::vector<uint32_t> all = g.tbits;
    all.insert(all.end(), g.cbits.begin(), g.cbits.end());
    const uint64_t ngroups = uint64_t(1) << (nq - all.size());
    if constexpr (sizeof(R) == 4 && K >= 3 && K <= 5) {
        if (dense_tc_applies(nq, g)) {  // complex64: tcgen05 with split TF32 operands
            launch_dense_tc(S.p, ns, nq, g, scratch, st);
            return true;
        }
    }
    // the tiled kernel where it measured faster than k_dense_dev on a 30-qubit state:
    // complex128 from K = 5 (17.3 vs 21.0 ms at K = 5; 10.8 vs 9.8 ms at K = 4), complex64,
    // whose compensated sums cost twice the FP64 ones, from K = 6 (42 vs 61 ms)
    if constexpr (K >= (sizeof(R) == 8 ? 5 : 6)) {
        using Sh = TiledShape<K>;
        if (ngroups >= (uint64_t)Sh::TG) {
            constexpr int D = Sh::D;
            std::vector<C<R>> mt((size_t)D * D);
            for (int r = 0; r < D; ++r)
                for (int c = 0; c < D; ++c) mt[(size_t)c * D + r] = cvt<R>(g.m[(size_t)r * D + c]);
            // pageable source: cudaMemcpyAsync stages it before returning
            B200SV_CUDA(cudaMemcpyAsync(scratch, mt.data(), mt.size() * sizeof(C<R>), cudaMemcpyHostToDevice, st));
            TiledP<R, K> p{};
            p.ins = make_insert(all);
            p.cmask = ctrl_mask(g.cbits);
            p.ntiles = ngroups / Sh::TG;
            fill_offsets(p.off, g.tbits);
            p.mt = static_cast<const C<R> *>(scratch);
            const int smem = (int)((kTileAmps + Sh::MSH) * sizeof(C<R>));
            B200SV_CUDA(cudaFuncSetAttribute(k_dense_tiled<R, K>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            const uint64_t grid = std::min<uint64_t>(p.ntiles, uint64_t(sm_count()) * 2);
            k_dense_tiled<R, K><<<dim3((unsigned)grid, ns), kTiledThreads, smem, st>>>(S, p);
            return true;
        }
        if constexpr (K > 6) return false;
    }
    if constexpr (sizeof(R) == 4 && K == 2) {
        const bool low2 = g.cbits.empty() && ((g.tbits[0] == 1 && g.tbits[1] == 0) || (g.tbits[0] == 0 && g.tbits[1] == 1));
        if (low2) {
            Dense2LowP<float> p{};
            p.ngroups = ngroups;
            for (int i = 0; i < 16; ++i) p.m[i] = cvt<float>(g.m[i]);
            if (g.tbits[0] == 0) k_dense2_low<true><<<grid_for(ngroups, ns), kThreads, 0, st>>>(S, p);
            else k_dense2_low<false><<<grid_for(ngroups, ns), kThreads, 0, st>>>(S, p);
            return true;
        }
    }
    if constexpr (K == 1) {
        if (g.cbits.empty() && g.tbits[0] == 0 && nq >= 5) {
            Dense1LowP<R> p{};
            p.n = uint64_t(1) << nq;
            for (int i = 0; i < 4; ++i) p.m[i] = cvt<R>(g.m[i]);
            k_dense1_low<R><<<grid_for(p.n, ns), kThreads, 0, st>>>(S, p);
            return true;
        }
    }
    if constexpr (K <= 4) {
        // the matrix as a kernel parameter (4^K entries; 4 KiB complex128 at K = 4): each
        // coefficient is a warp-uniform constant-bank operand, where a matrix in device memory
        // costs one L1 load per complex product
        DenseP<R, K> p{};
        p.ins = make_insert(all);
        p.cmask = ctrl_mask(g.cbits);
        p.ngroups = ngroups;
        fill_offsets(p.off, g.tbits);
        for (int i = 0; i < (1 << K) * (1 << K); ++i) p.m[i] = cvt<R>(g.m[i]);
        k_dense<R, K><<<grid_for(ngroups, ns, K == 1 ? 4 : 1), kThreads, 0, st>>>(S, p);
    } else if constexpr (K <= 6) {
        DenseDevP<R, K> p{};
        p.ins = make_insert(all);
        p.cmask = ctrl_mask(g.cbits);
        p.ngroups = ngroups;
        fill_offsets(p.off, g.tbits);
        std::vector<C<R>> hm(g.m.size());
        for (size_t i = 0; i < g.m.size(); ++i) hm[i] = cvt<R>(g.m[i]);
        // pageable source: cudaMemcpyAsync stages it before returning, so hm may go out of scope
        B200SV_CUDA(cudaMemcpyAsync(scratch, hm.data(), hm.size() * sizeof(C<R>), cudaMemcpyHostToDevice, st));
        p.m = static_cast<const C<R> *>(scratch);
        k_dense_dev<R, K><<<grid_for(ngroups, ns), kThreads, 0, st>>>(S, p);
    }
    return true;
}

template <typename R, int K>
void launch_diag_k(const States &S, int ns, uint32_t nq, const GateDesc &g, cudaStream_t st) {
    std::vector<uint32_t> all = g.tbits;
    all.insert(all.end(), g.cbits.begin(), g.cbits.end());
    DiagP<R, K> p{};
    p.ins = make_insert(all);
    p.cmask = ctrl_mask(g.cbits);
    p.ngroups = uint64_t(1) << (nq - all.size());
    fill_offsets(p.off, g.tbits);
    for (int i = 0; i < (1 << K); ++i) p.ph[i] = cvt<R>(g.m[i]);
    k_diag<R, K><<<grid_for(p.ngroups, ns, K >= 2 ? 2 : 4), kThreads, 0, st>>>(S, p);
}

template <typename R, int K>
void launch_pair_k(const States &S, int ns, uint32_t nq, const GateDesc &g, cudaStream_t st) {
    PairP<R, K> p{};
    p.ins = make_insert(g.tbits);
    p.ngroups = uint64_t(1) << (nq - g.tbits.size());
    fill_offsets(p.off, g.tbits);
    p.pa = (int)g.pa;
    p.pb = (int)g.pb;
    for (int i = 0; i < 4; ++i) p.m2[i] = cvt<R>(g.m2[i]);
    p.gamma = cvt<R>(g.gamma);
    p.scale_rest = (g.gamma != cd(1.0, 0.0)) ? 1 : 0;
    k_pair<R, K><<<grid_for(p.ngroups, ns), kThreads, 0, st>>>(S, p);
}

}  // namespace

template <typename R>
void launch_gate(void *const *states, int nstates, uint32_t nq, const GateDesc &g, void *scratch,
                 cudaStream_t st) {
    if (g.kind == Kind::Noop || nstates <= 0) return;
    if (nstates > kMaxStatesPerLaunch) throw ArgError("too many states in one launch");
    States S{};
    for (int i = 0; i < nstates; ++i) S.p[i] = states[i];
    const int nbits = (int)(g.tbits.size() + g.cbits.size());
    if (nbits > (int)nq) throw ArgError("gate acts on more wires than the state has");
    switch (g.kind) {
    case Kind::Dense:
        switch (g.k) {
        case 1: launch_dense_k<R, 1>(S, nstates, nq, g, scratch, st); break;
        case 2: launch_dense_k<R, 2>(S, nstates, nq, g, scratch, st); break;
        case 3: launch_dense_k<R, 3>(S, nstates, nq, g, scratch, st); break;
        case 4: launch_dense_k<R, 4>(S, nstates, nq, g, scratch, st); break;
        case 5: launch_dense_k<R, 5>(S, nstates, nq, g, scratch, st); break;
        case 6: launch_dense_k<R, 6>(S, nstates, nq, g, scratch, st); break;
        case 7:
        case 8:
        case 9:
        case 10: {
            bool done = false;
            switch (g.k) {
            case 7: done = launch_dense_k<R, 7>(S, nstates, nq, g, scratch, st); break;
            case 8: done = launch_dense_k<R, 8>(S, nstates, nq, g, scratch, st); break;
            case 9: done = launch_dense_k<R, 9>(S, nstates, nq, g, scratch, st); break;
            default: done = launch_dense_k<R, 10>(S, nstates, nq, g, scratch, st); break;
            }
            if (done) break;
        }
            [[fallthrough]];
        default: {
            if (g.k > 11 || !g.cbits.empty()) throw Unsupported("dense matrices act on at most 11 wires");
            BigDenseP p{};
            p.ins = make_insert(g.tbits);
            p.ngroups = uint64_t(1) << (nq - g.k);
            p.k = g.k;
            for (int j = 0; j < g.k; ++j) p.tmask[j] = uint64_t(1) << g.tbits[j];
            std::vector<C<R>> hm(g.m.size());
            for (size_t i = 0; i < g.m.size(); ++i) hm[i] = cvt<R>(g.m[i]);
            B200SV_CUDA(cudaMemcpyAsync(scratch, hm.data(), hm.size() * sizeof(C<R>), cudaMemcpyHostToDevice, st));
            const size_t sm = sizeof(C<R>) << g.k;
            if (sm > 48 * 1024)
                B200SV_CUDA(cudaFuncSetAttribute(k_dense_big<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            uint64_t nb = std::min<uint64_t>(p.ngroups, uint64_t(sm_count()) * 4);
            k_dense_big<R><<<dim3((unsigned)nb, nstates), kThreads, sm, st>>>(S, p, static_cast<const C<R> *>(scratch));
        }
        }
        break;
    case Kind::Diag:
        switch (g.k) {
        case 0: launch_diag_k<R, 0>(S, nstates, nq, g, st); break;
        case 1: launch_diag_k<R, 1>(S, nstates, nq, g, st); break;
        case 2: launch_diag_k<R, 2>(S, nstates, nq, g, st); break;
        default: throw Unsupported("diagonal form supports at most 2 target wires");
        }
        break;
    case Kind::Swap: {
        std::vector<uint32_t> all = g.tbits;
        all.insert(all.end(), g.cbits.begin(), g.cbits.end());
        SwapP p{};
        p.ins = make_insert(all);
        p.cmask = ctrl_mask(g.cbits);
        p.ngroups = uint64_t(1) << (nq - all.size());
        uint64_t off[8] = {};
        if (g.tbits.size() > 3) throw Unsupported("swap form supports at most 3 target wires");
        fill_offsets(off, g.tbits);
        p.oa = off[g.sa];
        p.ob = off[g.sb];
        k_swap<R><<<grid_for(p.ngroups, nstates, 4), kThreads, 0, st>>>(S, p);
        break;
    }
    case Kind::Pair:
        switch (g.k) {
        case 1: launch_pair_k<R, 1>(S, nstates, nq, g, st); break;
        case 2: launch_pair_k<R, 2>(S, nstates, nq, g, st); break;
        case 4: launch_pair_k<R, 4>(S, nstates, nq, g, st); break;
        default: throw Unsupported("pair form supports 1, 2 or 4 wires");
        }
        break;
    case Kind::Parity: {
        ParityP<R> p{};
        p.n = uint64_t(1) << nq;
        p.mask = g.pmask;
        p.ph[0] = cvt<R>(g.pphase[0]);
        p.ph[1] = cvt<R>(g.pphase[1]);
        k_parity<R><<<grid_for(p.n, nstates, 4), kThreads, 0, st>>>(S, p);
        break;
    }
    default: break;
    }
    B200SV_CUDA(cudaGetLastError());
}

template void launch_gate<float>(void *const *, int, uint32_t, const GateDesc &, void *, cudaStream_t);
template void launch_gate<double>(void *const *, int, uint32_t, const GateDesc &, void *, cudaStream_t);

}  // namespace b200sv
