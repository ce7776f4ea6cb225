// sv_noalloc.cu — Pauli-word expectation values that allocate nothing.
//
// Some callers cannot call cudaMalloc at the point where they need an
// expectation value: a serving loop whose device memory is owned by another
// allocator (PyTorch's caching allocator, a fixed arena), code that must not
// trigger cudaMalloc's implicit device synchronisation inside a latency budget,
// or a plugin host that forbids allocation after start-up.  For them
// b200sv_expval_pauli_noalloc evaluates <psi|P_t|psi> on a state the caller
// owns, writing into an output buffer the caller owns; its only scratch — the
// per-block partial sums of the two-pass reduction — is the file-scope array
// below.  Every GPU that loads this library holds that array (kScratchDoubles
// doubles, about 296 KiB) until the process exits.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  All calls share the one array, so
// calls that overlap on the GPU (different streams, or different host threads
// on the same device) race on it; serialise them.  Each launch writes every
// partial it later reads, so no clearing is needed between calls.
#include <mutex>
#include <string>
#include <vector>

#include "../../include/b200sv.h"
#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr int kNoAllocBlocks = 1184;  // partial sums per term (148 SMs x 8)
constexpr int kNoAllocThreads = 256;
constexpr size_t kScratchDoubles = size_t(kNoAllocBlocks) * B200SV_NOALLOC_MAX_TERMS;

static __device__ __align__(256) double g_noalloc_partials[kScratchDoubles];

std::mutex g_addr_mu;
std::vector<double *> g_addr;  // device address of g_noalloc_partials per device

double *scratch_address() {
    int dev = 0;
    B200SV_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if ((int)g_addr.size() <= dev) g_addr.resize(dev + 1, nullptr);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            throw CudaError(std::string("cudaGetSymbolAddress(g_noalloc_partials): ") + cudaGetErrorString(e));
        g_addr[dev] = static_cast<double *>(p);
    }
    return g_addr[dev];
}

// The state and the output must be device memory of the current device, where the
// scratch array's cached address is valid.  cudaPointerGetAttributes allocates nothing.
void check_on_current_device(const void *ptr, const char *what) {
    int dev = 0;
    B200SV_CUDA(cudaGetDevice(&dev));
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw ArgError(std::string("b200sv_expval_pauli_noalloc: ") + what + " is not a device pointer");
    }
    if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) || attr.device != dev)
        throw ArgError(std::string("b200sv_expval_pauli_noalloc: ") + what +
                       " must be device memory of the current device (" + std::to_string(dev) + ")");
}

struct WordsP {
    uint64_t xmask, hb_low, npairs;
    int nterms;
    uint64_t zmask[B200SV_NOALLOC_MAX_TERMS];
    int ny[B200SV_NOALLOC_MAX_TERMS];
};

// First pass: per-block partial sums of <psi|P_t|psi> for words sharing xmask.
template <typename R, int NT>
__global__ void __launch_bounds__(kNoAllocThreads) k_words(const C<R> *__restrict__ a, WordsP p, double *partials) {
    __shared__ double sm[NT * 32];
    double acc[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t] = 0.0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < p.npairs;
         g += (uint64_t)gridDim.x * blockDim.x) {
        if (p.xmask == 0) {
            const double2 z = widen<R>(a[g]);
            const double pr = z.x * z.x + z.y * z.y;
#pragma unroll
            for (int t = 0; t < NT; ++t)
                if (t < p.nterms) acc[t] += (__popcll(g & p.zmask[t]) & 1) ? -pr : pr;
        } else {
            const uint64_t lo = g & p.hb_low;
            const uint64_t i = ((g ^ lo) << 1) | lo;
            const double2 vi = widen<R>(a[i]), vj = widen<R>(a[i ^ p.xmask]);
            const double zr = vj.x * vi.x + vj.y * vi.y, zi = vj.x * vi.y - vj.y * vi.x;
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                if (t < p.nterms) {
                    const int q = p.ny[t] & 3;
                    double r = q == 0 ? zr : q == 1 ? -zi : q == 2 ? -zr : zi;
                    r *= 2.0;
                    acc[t] += (__popcll(i & p.zmask[t]) & 1) ? -r : r;
                }
            }
        }
    }
    block_reduce<NT>(acc, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int t = 0; t < NT; ++t)  // constant indices keep acc in registers
            if (t < p.nterms) partials[(size_t)t * gridDim.x + blockIdx.x] = acc[t];
    }
}

// Second pass: out[t] = sum_b partials[t, b] in a fixed order.
__global__ void k_words_finalize(const double *__restrict__ partials, int nb, double *__restrict__ out) {
    __shared__ double sm[32];
    double s[1] = {0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s[0] += partials[(size_t)blockIdx.x * nb + b];
    block_reduce<1>(s, sm);
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

template <typename R>
void launch_run(const void *state, uint32_t nq, const WordsP &p0, double *scratch, double *out, cudaStream_t st) {
    WordsP p = p0;
    const uint64_t n = uint64_t(1) << nq;
    if (p.xmask) {
        const int hb = 63 - __builtin_clzll(p.xmask);
        p.hb_low = (uint64_t(1) << hb) - 1;
        p.npairs = n / 2;
    } else {
        p.hb_low = 0;
        p.npairs = n;
    }
    uint64_t nb = (p.npairs + kNoAllocThreads * 4 - 1) / (kNoAllocThreads * 4);
    nb = std::max<uint64_t>(1, std::min<uint64_t>(nb, kNoAllocBlocks));
    const C<R> *a = static_cast<const C<R> *>(state);
    if (p.nterms == 1) k_words<R, 1><<<(unsigned)nb, kNoAllocThreads, 0, st>>>(a, p, scratch);
    else if (p.nterms <= 8) k_words<R, 8><<<(unsigned)nb, kNoAllocThreads, 0, st>>>(a, p, scratch);
    else k_words<R, B200SV_NOALLOC_MAX_TERMS><<<(unsigned)nb, kNoAllocThreads, 0, st>>>(a, p, scratch);
    B200SV_CUDA(cudaGetLastError());
    k_words_finalize<<<p.nterms, 128, 0, st>>>(scratch, (int)nb, out);
    B200SV_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace b200sv

using namespace b200sv;

extern "C" int b200sv_expval_pauli_noalloc(const void *state_device, uint32_t num_qubits, int dtype, uint32_t nterms,
                                           const uint32_t *offsets, const uint32_t *wires, const char *paulis,
                                           double *out_device, void *cuda_stream) {
    return run_guarded([&] {
        if (!state_device || !out_device) throw ArgError("b200sv_expval_pauli_noalloc: NULL state or output pointer");
        if (dtype != B200SV_C64 && dtype != B200SV_C128) throw ArgError("b200sv_expval_pauli_noalloc: bad dtype");
        if (num_qubits < 1 || num_qubits > 36)
            throw ArgError("b200sv_expval_pauli_noalloc: number of qubits must be in [1, 36]");
        if (nterms > B200SV_NOALLOC_MAX_TERMS)
            throw ArgError("b200sv_expval_pauli_noalloc: at most " + std::to_string(B200SV_NOALLOC_MAX_TERMS) +
                           " Pauli words per call (got " + std::to_string(nterms) + ")");
        check_on_current_device(state_device, "state_device");
        check_on_current_device(out_device, "out_device");
        if (nterms == 0) return;
        if (!offsets) throw ArgError("b200sv_expval_pauli_noalloc: NULL offsets");
        // Words, validated on the host (no device memory involved).
        std::vector<uint64_t> xm(nterms), zm(nterms);
        std::vector<int> ny(nterms);
        for (uint32_t t = 0; t < nterms; ++t) {
            if (offsets[t] > offsets[t + 1]) throw ArgError("b200sv_expval_pauli_noalloc: offsets must not decrease");
            uint64_t used = 0;
            xm[t] = zm[t] = 0;
            ny[t] = 0;
            for (uint32_t q = offsets[t]; q < offsets[t + 1]; ++q) {
                if (!wires || !paulis) throw ArgError("b200sv_expval_pauli_noalloc: NULL wires or paulis");
                if (wires[q] >= num_qubits) throw ArgError("b200sv_expval_pauli_noalloc: wire out of range");
                const uint64_t bit = uint64_t(1) << (num_qubits - 1 - wires[q]);
                if (used & bit) throw ArgError("All wires in observables must be disjoint.");
                used |= bit;
                switch (paulis[q]) {
                case 'I': break;
                case 'X': xm[t] |= bit; break;
                case 'Y': xm[t] |= bit; zm[t] |= bit; ny[t]++; break;
                case 'Z': zm[t] |= bit; break;
                default: throw ArgError("Pauli letters must be I, X, Y or Z");
                }
            }
        }
        double *scratch = scratch_address();
        cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
        // consecutive words with equal X masks share one pass; runs are launched in order
        for (uint32_t t0 = 0; t0 < nterms;) {
            uint32_t t1 = t0 + 1;
            while (t1 < nterms && xm[t1] == xm[t0]) ++t1;
            WordsP p{};
            p.xmask = xm[t0];
            p.nterms = (int)(t1 - t0);
            for (uint32_t t = t0; t < t1; ++t) {
                p.zmask[t - t0] = zm[t];
                p.ny[t - t0] = ny[t];
            }
            if (dtype == B200SV_C64) launch_run<float>(state_device, num_qubits, p, scratch, out_device + t0, st);
            else launch_run<double>(state_device, num_qubits, p, scratch, out_device + t0, st);
            t0 = t1;
        }
    });
}
