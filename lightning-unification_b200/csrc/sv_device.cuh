// sv_device.cuh — device-side building blocks shared by every kernel of libb200sv.
//
// State layout in HBM: one contiguous array of 2^n amplitudes, interleaved
// (re, im) as float2 (complex64) or double2 (complex128); basis index bit
// (n-1-w) holds wire w, so wire 0 is the most significant bit, as in
// lightning.qubit (LQ/gates/cpu_kernels/GateImplementationsLM.hpp:210).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace b200sv {

template <typename R> struct cvec;
template <> struct cvec<double> { using type = double2; };
template <> struct cvec<float> { using type = float2; };
template <typename R> using C = typename cvec<R>::type;

template <typename R> __host__ __device__ __forceinline__ C<R> mk(R re, R im) {
    C<R> z; z.x = re; z.y = im; return z;
}
template <typename R> __device__ __forceinline__ C<R> cmul(C<R> a, C<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ---- bit insertion -------------------------------------------------------
// A gate on k target (+c control) bits visits 2^(n-k-c) groups.  Group index g
// is spread over the non-gate bits by inserting a zero at every gate bit
// position, lowest position first (the revWireParity scheme of
// GateImplementationsLM.hpp:51-125, generalised to any number of bits).
constexpr int kMaxInsert = 16;
struct Insert {
    int nb;
    uint64_t low[kMaxInsert];  // (1 << pos_j) - 1 for ascending positions pos_j
    __device__ __forceinline__ uint64_t operator()(uint64_t g) const {
#pragma unroll
        for (int j = 0; j < kMaxInsert; ++j) {
            if (j < nb) {
                const uint64_t lo = g & low[j];
                g = ((g ^ lo) << 1) | lo;
            }
        }
        return g;
    }
};

// ---- accumulation policies ---------------------------------------------
// complex128: plain FMA chains.
// complex64: compensated dot products in FP32 pairs — every product is split
// exactly with an FMA (TwoProduct) and every addition with Knuth's TwoSum; the
// error terms are summed separately and added once at the end.  This is the
// Dot2 algorithm of Ogita, Rump and Oishi, "Accurate sum and dot product",
// SIAM J. Sci. Comput. 26(6), 2005; the result is as accurate as if computed in
// twice the working precision and then rounded once.
template <typename R> struct Acc;
template <> struct Acc<double> {
    double s = 0.0;
    __device__ __forceinline__ void add_prod(double a, double b) { s = fma(a, b, s); }
    __device__ __forceinline__ double get() const { return s; }
};
template <> struct Acc<float> {
    float s = 0.0f, c = 0.0f;
    __device__ __forceinline__ void add_prod(float a, float b) {
        const float p = a * b;
        const float ep = fmaf(a, b, -p);  // exact: a*b = p + ep
        const float t = s + p;            // TwoSum(s, p) = t + et
        const float z = t - s;
        const float et = (s - (t - z)) + (p - z);
        s = t;
        c += ep + et;
    }
    __device__ __forceinline__ float get() const { return s + c; }
};

// out = sum_j m_j * v_j for complex m, v with the precision policy of R.
template <typename R> struct CAcc {
    Acc<R> re, im;
    __device__ __forceinline__ void add(C<R> m, C<R> v) {
        re.add_prod(m.x, v.x);
        re.add_prod(-m.y, v.y);
        im.add_prod(m.x, v.y);
        im.add_prod(m.y, v.x);
    }
    __device__ __forceinline__ C<R> get() const { return mk<R>(re.get(), im.get()); }
};

// ---- deterministic FP64 block reduction -----------------------------------
// Shuffle-down tree inside each warp, then warp totals tree-reduced by warp 0.
// The association order depends only on blockDim, so results are reproducible
// run to run.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double *smem /* NV*32 */) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? smem[k * 32 + lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
            v[k] = x;
        }
    }
    __syncthreads();
}

// widen an amplitude to FP64 for reductions
template <typename R> __device__ __forceinline__ double2 widen(C<R> a) {
    return make_double2((double)a.x, (double)a.y);
}

}  // namespace b200sv
