// sv_sparse.cu — expectation value and variance of a sparse Hamiltonian given in CSR form.
//
// The reference forms the whole vector y = H psi with a sequential CSR product
// (LQ/utils/SparseLinAlg.hpp:43-62) and then takes innerProdC(psi, y) for the
// expectation value and innerProdC(y, y) - Re(innerProdC(y, psi))^2 for the variance
// (LQ/measurements/MeasurementsLQubit.hpp:197-214, :451-472).  Here each row's y_i is
// formed in registers by a group of W lanes and folded straight into the two FP64
// sums Re(conj(psi_i) y_i) and |y_i|^2, so y is never written to memory; both values
// come out of one read of the CSR arrays and of the state.
//
// Row i owns the non-zeros [row_map[i] - row_map[0], row_map[i+1] - row_map[0]),
// which is the reference's sequential cursor over the value array.
#include <algorithm>

#include "sv_device.cuh"
#include "sv_internal.hpp"

namespace b200sv {
namespace {

constexpr int kST = 256;

// The CSR arrays are checked here, on the device, as they are read: a row whose bounds are
// decreasing (or below row_map[0]) sets bit 0 of *bad, one ending past the `used` entries
// sets bit 2, and either counts as empty; a column index outside the state sets bit 1 and
// its term is skipped, so no access leaves the arrays.  The host turns the bits into the
// error messages of the host-array checks.
template <typename R, int W>
__global__ void __launch_bounds__(kST) k_sparse_ev(const C<R> *__restrict__ psi, const uint64_t *__restrict__ row_map,
                                                   const uint64_t *__restrict__ cols, const C<R> *__restrict__ vals,
                                                   uint64_t nrows, uint64_t used, double *partials,
                                                   unsigned int *bad) {
    __shared__ double sm[2 * 32];
    double acc[2] = {0.0, 0.0};
    const int lane = threadIdx.x % W;
    const uint64_t base = row_map[0];
    const uint64_t groups = (uint64_t)gridDim.x * (blockDim.x / W);
    // r0 is the same for all lanes of a warp, so every lane makes the same number of
    // trips and reaches every shuffle
    const uint64_t warp_row0 = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / 32) * (32 / W);
    for (uint64_t r0 = warp_row0; r0 < nrows; r0 += groups) {
        const uint64_t r = r0 + (threadIdx.x % 32) / W;
        const bool live = r < nrows;
        double yr = 0.0, yi = 0.0;
        if (live) {
            const uint64_t lo = row_map[r], hi = row_map[r + 1];
            uint64_t b = lo - base, e = hi - base;
            if (hi < lo || lo < base || e > used) {
                if (lane == 0) atomicOr(bad, e > used && hi >= lo && lo >= base ? 4u : 1u);
                e = b = 0;
            }
            for (uint64_t k = b + lane; k < e; k += W) {
                const uint64_t c = cols[k];
                if (c >= nrows) {
                    atomicOr(bad, 2u);
                    continue;
                }
                const double2 v = widen<R>(vals[k]);
                const double2 x = widen<R>(psi[c]);
                yr = fma(v.x, x.x, fma(-v.y, x.y, yr));
                yi = fma(v.x, x.y, fma(v.y, x.x, yi));
            }
        }
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) {
            yr += __shfl_xor_sync(0xffffffffu, yr, o, W);
            yi += __shfl_xor_sync(0xffffffffu, yi, o, W);
        }
        if (live && lane == 0) {
            const double2 p = widen<R>(psi[r]);
            acc[0] += p.x * yr + p.y * yi;  // Re conj(psi_r) y_r
            acc[1] += yr * yr + yi * yi;    // |y_r|^2
        }
    }
    block_reduce<2>(acc, sm);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = acc[0];
        partials[gridDim.x + blockIdx.x] = acc[1];
    }
}

__global__ void k_sparse_finalize(const double *__restrict__ partials, int nb, double *__restrict__ out) {
    __shared__ double sm[2 * 32];
    double s[2] = {0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        s[0] += partials[b];
        s[1] += partials[nb + b];
    }
    block_reduce<2>(s, sm);
    if (threadIdx.x == 0) {
        out[0] = s[0];
        out[1] = s[1];
    }
}

template <typename R, int W>
void launch_w(const void *psi, const uint64_t *row_map, const uint64_t *cols, const void *vals, uint64_t nrows,
              uint64_t used, double *partials, unsigned int *bad, int nb, cudaStream_t st) {
    k_sparse_ev<R, W><<<nb, kST, 0, st>>>(static_cast<const C<R> *>(psi), row_map, cols,
                                          static_cast<const C<R> *>(vals), nrows, used, partials, bad);
}

}  // namespace

// Lanes per row: the power of two nearest the mean row length, at most a warp.
int sparse_lanes(uint64_t nrows, uint64_t nnz) {
    const double mean = nrows ? double(nnz) / double(nrows) : 0.0;
    int w = 1;
    while (w < 32 && 2.0 * w <= mean) w *= 2;
    return w;
}

template <typename R>
void reduce_sparse(const void *psi, uint32_t nq, const uint64_t *row_map_dev, const uint64_t *cols_dev,
                   const void *vals_dev, uint64_t nnz, double *partials, double *out_dev, unsigned int *bad_dev,
                   cudaStream_t st) {
    const uint64_t nrows = uint64_t(1) << nq;
    const int w = sparse_lanes(nrows, nnz);
    const uint64_t threads = nrows * (uint64_t)w;
    const int nb = (int)std::max<uint64_t>(1, std::min<uint64_t>((threads + kST - 1) / kST, kMaxRedBlocks));
    const uint64_t *rm = row_map_dev, *cl = cols_dev;
    switch (w) {
    case 1: launch_w<R, 1>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    case 2: launch_w<R, 2>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    case 4: launch_w<R, 4>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    case 8: launch_w<R, 8>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    case 16: launch_w<R, 16>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    default: launch_w<R, 32>(psi, rm, cl, vals_dev, nrows, nnz, partials, bad_dev, nb, st); break;
    }
    B200SV_CUDA(cudaGetLastError());
    k_sparse_finalize<<<1, 128, 0, st>>>(partials, nb, out_dev);
    B200SV_CUDA(cudaGetLastError());
}

template void reduce_sparse<float>(const void *, uint32_t, const uint64_t *, const uint64_t *, const void *,
                                   uint64_t, double *, double *, unsigned int *, cudaStream_t);
template void reduce_sparse<double>(const void *, uint32_t, const uint64_t *, const uint64_t *, const void *,
                                    uint64_t, double *, double *, unsigned int *, cudaStream_t);

}  // namespace b200sv
