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

dim3 grid_for(uint64_t work, int nstates) {
    const uint64_t cap = uint64_t(sm_count()) * 16;
    uint64_t b = (work + kThreads - 1) / kThreads;
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
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g) | p.cmask;
        C<R> v[D];
#pragma unroll
        for (int r = 0; r < D; ++r) v[r] = sv[base + p.off[r]];
#pragma unroll
        for (int r = 0; r < D; ++r) {
            CAcc<R> a;
#pragma unroll
            for (int c = 0; c < D; ++c) a.add(p.m[r * D + c], v[c]);
            sv[base + p.off[r]] = a.get();
        }
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
        for (int r = 0; r < D; ++r) {
            CAcc<R> a;
#pragma unroll
            for (int c = 0; c < D; ++c) a.add(__ldg(&p.m[r * D + c]), v[c]);
            sv[base + p.off[r]] = a.get();
        }
    }
}

// Large dense blocks (k = 7..11): one CTA per group, the group staged in shared memory.
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
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g) | p.cmask;
#pragma unroll
        for (int r = 0; r < (1 << K); ++r) {
            const C<R> v = sv[base + p.off[r]];
            CAcc<R> a;
            a.add(p.ph[r], v);
            sv[base + p.off[r]] = a.get();
        }
    }
}

struct SwapP {
    Insert ins;
    uint64_t cmask, ngroups, oa, ob;
};
template <typename R>
__global__ void __launch_bounds__(kThreads) k_swap(States s, SwapP p) {
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = p.ins(g) | p.cmask;
        const C<R> a = sv[base + p.oa];
        const C<R> b = sv[base + p.ob];
        sv[base + p.oa] = b;
        sv[base + p.ob] = a;
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
    C<R> *__restrict__ sv = static_cast<C<R> *>(s.p[blockIdx.y]);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < p.n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const C<R> v = sv[i];
        CAcc<R> a;
        a.add(p.ph[__popcll(i & p.mask) & 1], v);
        sv[i] = a.get();
    }
}

template <typename R> C<R> cvt(const cd &z) { return mk<R>((R)z.real(), (R)z.imag()); }

template <typename R, int K>
void launch_dense_k(const States &S, int ns, uint32_t nq, const GateDesc &g, void *scratch,
                    cudaStream_t st) {
    std::vector<uint32_t> all = g.tbits;
    all.insert(all.end(), g.cbits.begin(), g.cbits.end());
    const uint64_t ngroups = uint64_t(1) << (nq - all.size());
    if constexpr (K <= 3) {
        DenseP<R, K> p{};
        p.ins = make_insert(all);
        p.cmask = ctrl_mask(g.cbits);
        p.ngroups = ngroups;
        fill_offsets(p.off, g.tbits);
        for (int i = 0; i < (1 << K) * (1 << K); ++i) p.m[i] = cvt<R>(g.m[i]);
        k_dense<R, K><<<grid_for(ngroups, ns), kThreads, 0, st>>>(S, p);
    } else {
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
    k_diag<R, K><<<grid_for(p.ngroups, ns), kThreads, 0, st>>>(S, p);
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
        k_swap<R><<<grid_for(p.ngroups, nstates), kThreads, 0, st>>>(S, p);
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
        k_parity<R><<<grid_for(p.n, nstates), kThreads, 0, st>>>(S, p);
        break;
    }
    default: break;
    }
    B200SV_CUDA(cudaGetLastError());
}

template void launch_gate<float>(void *const *, int, uint32_t, const GateDesc &, void *, cudaStream_t);
template void launch_gate<double>(void *const *, int, uint32_t, const GateDesc &, void *, cudaStream_t);

}  // namespace b200sv
