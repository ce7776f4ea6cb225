// sv_tensor.cu — complex64 dense k-wire matrices (k = 3..5) on the 5th-generation tensor cores.
//
// applyMatrix of a 2^k x 2^k complex matrix U on k target wires is, per group g of the
// state (the 2^k amplitudes that differ only in the target bits), y_g = U x_g.  Stacking
// 128 groups as rows and writing each amplitude as its (re, im) pair gives a real GEMM
//     Y[128 x 2D] = X[128 x 2D] . W[2D x 2D],   D = 2^k,
// with W[2c+a][2r+b] the real embedding of U: W[2c][2r] = W[2c+1][2r+1] = Re U[r][c],
// W[2c+1][2r] = -Im U[r][c], W[2c][2r+1] = Im U[r][c].  Each CTA tile runs it with
// tcgen05.mma kind::tf32 (operands in shared memory, the 128 x 2D FP32 accumulator in
// tensor memory), and the epilogue reads the accumulator back with tcgen05.ld and stores
// the amplitudes in place.
//
// Precision: TF32 keeps 10 explicit mantissa bits, so both operands are split, x = x_hi +
// x_lo with x_hi = x rounded to TF32 and x_lo = x - x_hi (exact in FP32), and the product is
// accumulated as hi.hi + hi.lo + lo.hi in FP32 in tensor memory (the split-operand scheme of
// Ootomo and Yokota, "Recovering single precision accuracy from Tensor Cores while surpassing
// the FP32 theoretical peak performance", IJHPCA 2022; the dropped lo.lo term is below
// 2^-22 of each product).  Results are FP32-accurate sums of 2D products, not the
// compensated sums of the CUDA-core kernels.
//
// Shared-memory operands use the no-swizzle K-major canonical layout: 8 rows x 16 bytes
// "core matrices", contiguous, the next core matrix along K 128 bytes further (leading
// byte offset) and the next 8 rows (KK / 4) x 128 bytes further (stride byte offset).
// One MMA consumes K = 8 TF32 values (two core matrices along K).
//
// The only wait is on the MMA-completion mbarrier; it gives up after a bounded number of
// polls, counts the failure in g_tc_timeouts (reported by b200sv_synchronize) and the CTA
// still releases its tensor memory.
#include <algorithm>
#include <cstring>
#include <vector>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {

__device__ unsigned int g_tc_timeouts = 0;

namespace {

constexpr int kTcM = 128;        // rows (groups) per tile: the MMA's M
constexpr int kTcThreads = 128;  // thread t owns row t (tensor-memory lane t)
constexpr int kTcMaxK = 5;

struct TcStates {
    void *p[kMaxStatesPerLaunch];
};

struct TcP {
    Insert ins;         // group index -> base index (zeros at the target bits)
    uint64_t ntiles;    // groups / 128
    uint64_t off[1 << kTcMaxK];  // offset of row r of a group (bit k-1-j of r <-> target j)
    const float *b;     // W^T split, in the shared-memory layout: hi (2D x 2D) then lo
};

// byte offset of element (row, col) in the K-major no-swizzle layout of a matrix with KK columns
__host__ __device__ constexpr uint32_t core_off(uint32_t row, uint32_t col, uint32_t KK) {
    return ((row >> 3) * (KK >> 2) + (col >> 2)) * 128u + (row & 7u) * 16u + (col & 3u) * 4u;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start >> 4, leading byte offset >> 4 (bits 16..29),
// stride byte offset >> 4 (bits 32..45), descriptor version 1 (bit 46), no swizzle (bits 61..63 = 0)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// instruction descriptor of kind::tf32: F32 accumulator (bits 4..5 = 1), A and B TF32 (bits
// 7..9 and 10..12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits 17..22, M >> 4 at 24..28
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[NC]);
template <> __device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int K>
__global__ void __launch_bounds__(kTcThreads) k_dense_tc(TcStates s, TcP p) {
    constexpr int D = 1 << K, KK = 2 * D, NN = 2 * D;
    constexpr uint32_t kCols = NN < 32 ? 32 : NN;  // tensor-memory columns (a power of two >= 32)
    constexpr uint32_t kA = kTcM * KK * 4, kB = NN * KK * 4;  // bytes of one split operand
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sa_hi = smem, *sa_lo = smem + kA, *sb_hi = smem + 2 * kA, *sb_lo = smem + 2 * kA + kB;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t s_tmem;
    float2 *sv = static_cast<float2 *>(s.p[blockIdx.y]);
    const int warp = threadIdx.x >> 5;

    // the split W^T, prepared on the host in the shared-memory layout
    {
        const float4 *src = reinterpret_cast<const float4 *>(p.b);
        float4 *dst = reinterpret_cast<float4 *>(sb_hi);
        for (uint32_t i = threadIdx.x; i < 2 * kB / 16; i += kTcThreads) dst[i] = src[i];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    constexpr uint32_t idesc = idesc_tf32(kTcM, NN);
    constexpr uint32_t kLbo = 128, kSboA = (KK / 4) * 128, kSboB = (KK / 4) * 128;
    uint32_t phase = 0;
    bool ok = true;

    // Software pipeline: the amplitudes of the thread's next row are loaded into registers while
    // the MMAs and the epilogue of the current tile run (tiles are disjoint sets of amplitudes).
    float2 x[D];
    uint64_t t = blockIdx.x;
    uint64_t base = 0;
    if (t < p.ntiles) {
        base = p.ins(t * kTcM + threadIdx.x);
#pragma unroll
        for (int c = 0; c < D; ++c) x[c] = sv[base + p.off[c]];
    }
    for (; t < p.ntiles && ok; t += gridDim.x) {
        // row threadIdx.x: split and store to the operand layouts
#pragma unroll
        for (int c = 0; c < D; ++c) {
            const float hx = tf32_rna(x[c].x), hy = tf32_rna(x[c].y);
            const uint32_t o = core_off(threadIdx.x, 2 * c, KK);
            *reinterpret_cast<float2 *>(sa_hi + o) = make_float2(hx, hy);
            *reinterpret_cast<float2 *>(sa_lo + o) = make_float2(x[c].x - hx, x[c].y - hy);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_hi = smem_u32(sa_hi), a_lo = smem_u32(sa_lo);
            const uint32_t b_hi = smem_u32(sb_hi), b_lo = smem_u32(sb_lo);
#pragma unroll
            for (int pass = 0; pass < 3; ++pass) {
                const uint32_t a = pass == 2 ? a_lo : a_hi, b = pass == 1 ? b_lo : b_hi;
#pragma unroll
                for (int ks = 0; ks < KK / 8; ++ks)
                    mma_tf32(tmem, smem_desc(a + ks * 256, kLbo, kSboA), smem_desc(b + ks * 256, kLbo, kSboB),
                             idesc, (pass | ks) != 0 ? 1u : 0u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        // the next tile's row, in flight during the MMAs and the epilogue
        const uint64_t cur = base;
        const uint64_t tn = t + gridDim.x;
        if (tn < p.ntiles) {
            base = p.ins(tn * kTcM + threadIdx.x);
#pragma unroll
            for (int c = 0; c < D; ++c) x[c] = sv[base + p.off[c]];
        }
        // wait for the MMAs (bounded)
        uint32_t done = 0;
        for (uint32_t it = 0; it < (1u << 22) && !done; ++it) {
            asm volatile(
                "{\n\t.reg .pred q;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, q;\n\t}"
                : "=r"(done)
                : "r"(smem_u32(&mbar)), "r"(phase)
                : "memory");
        }
        phase ^= 1u;
        // block-uniform decision: the epilogue's tcgen05.ld is a warp-wide (.sync.aligned) instruction
        if (__syncthreads_and(done ? 1 : 0) == 0) {
            if (threadIdx.x == 0) atomicAdd(&g_tc_timeouts, 1u);
            ok = false;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (ok) {
            const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
            for (int chunk = 0; chunk < NN / 16; ++chunk) {
                float v[16];
                tmem_ld<16>(lane_base + chunk * 16, v);
#pragma unroll
                for (int j = 0; j < 8; ++j) sv[cur + p.off[chunk * 8 + j]] = make_float2(v[2 * j], v[2 * j + 1]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // operands and accumulator free for the next tile
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// TF32 rounding (nearest, ties away from zero) of an FP32 value, as cvt.rna.tf32.f32
float tf32_host(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & 0xFFFFE000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

template <int K>
void launch_tc(float2 *const *states, int ns, uint32_t nq, const GateDesc &g, void *scratch, cudaStream_t st) {
    constexpr int D = 1 << K, KK = 2 * D, NN = 2 * D;
    // W^T[n][kk] = W[kk][n], split into TF32 hi and lo parts, in the operand layout
    std::vector<unsigned char> blob(2 * (size_t)NN * KK * 4, 0);
    auto put = [&](int part, int n, int kk, float v) {
        std::memcpy(blob.data() + (size_t)part * NN * KK * 4 + core_off(n, kk, KK), &v, 4);
    };
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) {
            const float ur = (float)g.m[(size_t)r * D + c].real(), ui = (float)g.m[(size_t)r * D + c].imag();
            // W[2c+a][2r+b]: (0,0) Re, (1,0) -Im, (0,1) Im, (1,1) Re  ->  W^T[2r+b][2c+a]
            const float w[2][2] = {{ur, -ui}, {ui, ur}};  // [b][a]
            for (int bb = 0; bb < 2; ++bb)
                for (int aa = 0; aa < 2; ++aa) {
                    const float x = w[bb][aa], hi = tf32_host(x), lo = x - hi;
                    put(0, 2 * r + bb, 2 * c + aa, hi);
                    put(1, 2 * r + bb, 2 * c + aa, lo);
                }
        }
    // pageable source: cudaMemcpyAsync stages it before returning
    B200SV_CUDA(cudaMemcpyAsync(scratch, blob.data(), blob.size(), cudaMemcpyHostToDevice, st));
    TcP p{};
    std::vector<uint32_t> bits = g.tbits;
    std::sort(bits.begin(), bits.end());
    p.ins.nb = K;
    for (int j = 0; j < K; ++j) p.ins.low[j] = (uint64_t(1) << bits[j]) - 1;
    p.ntiles = (uint64_t(1) << (nq - K)) / kTcM;
    for (int r = 0; r < D; ++r) {
        uint64_t o = 0;
        for (int j = 0; j < K; ++j)
            if (r & (1 << (K - 1 - j))) o |= uint64_t(1) << g.tbits[j];
        p.off[r] = o;
    }
    p.b = static_cast<const float *>(scratch);
    const int smem = 2 * (kTcM * KK * 4) + 2 * (NN * KK * 4);
    B200SV_CUDA(cudaFuncSetAttribute(k_dense_tc<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int per_sm = K == 3 ? 12 : K == 4 ? 5 : 2;  // CTAs that fit an SM's shared memory
    const uint64_t grid = std::min<uint64_t>(p.ntiles, (uint64_t)sm_count() * per_sm);
    TcStates S{};
    for (int i = 0; i < ns; ++i) S.p[i] = states[i];
    k_dense_tc<K><<<dim3((unsigned)grid, ns), kTcThreads, smem, st>>>(S, p);
    B200SV_CUDA(cudaGetLastError());
}

}  // namespace

size_t dense_tc_scratch_bytes(int k) { return k >= 3 && k <= kTcMaxK ? (size_t)2 * (2 << k) * (2 << k) * 4 : 0; }

bool dense_tc_applies(uint32_t nq, const GateDesc &g) {
    return g.kind == Kind::Dense && g.k >= 3 && g.k <= kTcMaxK && g.cbits.empty() &&
           nq >= (uint32_t)g.k + 7;  // at least one 128-row tile
}

void launch_dense_tc(void *const *states, int ns, uint32_t nq, const GateDesc &g, void *scratch, cudaStream_t st) {
    float2 *const *s = reinterpret_cast<float2 *const *>(states);
    switch (g.k) {
    case 3: launch_tc<3>(s, ns, nq, g, scratch, st); break;
    case 4: launch_tc<4>(s, ns, nq, g, scratch, st); break;
    case 5: launch_tc<5>(s, ns, nq, g, scratch, st); break;
    default: throw Unsupported("tensor-core dense path covers 3..5 wires");
    }
}

unsigned int dense_tc_timeouts() {
    unsigned int v = 0;
    B200SV_CUDA(cudaMemcpyFromSymbol(&v, g_tc_timeouts, sizeof(v)));
    return v;
}

}  // namespace b200sv
