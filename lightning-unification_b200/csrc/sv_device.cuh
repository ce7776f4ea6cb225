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
// complex64: each output is a compensated sum in FP32 pairs (value, error).
// Every complex product term is formed with one FMA per component
// (re = fma(a.x, b.x, -a.y*b.y), im = fma(a.x, b.y, a.y*b.x)), and the terms are
// added with Knuth's TwoSum (D. E. Knuth, TAOCP vol. 2, 4.2.2), whose rounding
// errors are carried in a second FP32 word and added once at the end — the
// summation half of the Dot2 scheme of Ogita, Rump and Oishi, "Accurate sum and
// dot product", SIAM J. Sci. Comput. 26(6), 2005.
template <typename R> struct CAcc;
template <> struct CAcc<double> {
    double re = 0.0, im = 0.0;
    __device__ __forceinline__ void add(double2 m, double2 v) {
        re = fma(m.x, v.x, re);
        re = fma(-m.y, v.y, re);
        im = fma(m.x, v.y, im);
        im = fma(m.y, v.x, im);
    }
    __device__ __forceinline__ double2 get() const { return make_double2(re, im); }
    // the first term of a sum: the same value as add() on an empty accumulator
    __device__ __forceinline__ void set(double2 m, double2 v) {
        re = 0.0;
        im = 0.0;
        add(m, v);
    }
};
__device__ __forceinline__ void two_sum_acc(float &s, float &c, float t) {
    const float u = s + t;
    const float z = u - s;
    c += (s - (u - z)) + (t - z);
    s = u;
}
// Paired FP32 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2): the real and imaginary parts go
// through one instruction each step, with the same rounded operations per component as the
// scalar forms, so results are bit-identical to them.
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
// complex product m * v with FMA-formed components:
// (fma(m.x, v.x, -(m.y v.y)), fma(m.x, v.y, m.y v.x))
__device__ __forceinline__ float2 cmul2(float2 m, float2 v) {
    const float2 q = __fmul2_rn(make_float2(m.y, m.y), make_float2(v.y, v.x));
    return __ffma2_rn(make_float2(m.x, m.x), v, make_float2(-q.x, q.y));
}
// two_sum_acc on both components at once
__device__ __forceinline__ void two_sum_acc2(float2 &s, float2 &c, float2 t) {
    const float2 u = __fadd2_rn(s, t);
    const float2 z = sub2(u, s);
    c = __fadd2_rn(c, __fadd2_rn(sub2(s, sub2(u, z)), sub2(t, z)));
    s = u;
}
template <> struct CAcc<float> {
    float2 s = make_float2(0.0f, 0.0f), c = make_float2(0.0f, 0.0f);
    __device__ __forceinline__ void add(float2 m, float2 v) { two_sum_acc2(s, c, cmul2(m, v)); }
    __device__ __forceinline__ float2 get() const { return __fadd2_rn(s, c); }
    // the first term of a sum: TwoSum with an empty accumulator is exact (value t, error 0),
    // so the term is stored directly — the same value as add() without its six additions
    __device__ __forceinline__ void set(float2 m, float2 v) {
        s = cmul2(m, v);
        c = make_float2(0.0f, 0.0f);
    }
};
// term c of a sum formed in a loop unrolled at compile time: the first term starts the sum
template <typename R>
__device__ __forceinline__ void cacc_term(CAcc<R> &a, int c, C<R> m, C<R> v) {
    if (c == 0) a.set(m, v);
    else a.add(m, v);
}

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

// ---- asynchronous global -> shared copies (16 bytes, both addresses 16-byte aligned) ----
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// widen an amplitude to FP64 for reductions
template <typename R> __device__ __forceinline__ double2 widen(C<R> a) {
    return make_double2((double)a.x, (double)a.y);
}

}  // namespace b200sv
