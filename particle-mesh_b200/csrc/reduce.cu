// FP64 reductions of the step's conserved quantities: the total mass on the
// mesh, sum over cells of (delta + 1), and the total momentum m sum_p v_p.
// The FP32 path keeps FP64 for these sums (with 1.07e9 cells or 1.3e8
// particles an FP32 running sum loses every digit of a 1e-7 drift).  No
// counterpart in the reference, which does no conservation diagnostics.
//
// Deterministic: a fixed grid, each block's partial sums in a fixed tree
// order into a plan-owned scratch array, then one block adds the partials in
// block order, so repeated calls on the same data give identical bits.
#include "pm_internal.cuh"

namespace pmb {

namespace {

constexpr int kRedThreads = 256;

// v summed over the block (every thread returns the same total).
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    return t;
}

// partial[4 * block + c]: c = 0 the mesh total, 1..3 the momentum components
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_reduce_partials(const T* __restrict__ mesh, int n,
                                                                 const T* __restrict__ vx,
                                                                 const T* __restrict__ vy,
                                                                 const T* __restrict__ vz, long long np,
                                                                 double* __restrict__ partial) {
    __shared__ double sh[kRedThreads / 32];
    double m = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    if (mesh) {
        const long long cells = (long long)n * n * n;
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
             c += (long long)gridDim.x * blockDim.x) {
            const long long row = c / n;
            m += (double)mesh[row * (n + 2) + (c - row * n)] + 1.0;
        }
    }
    if (vx) {
        for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
             p += (long long)gridDim.x * blockDim.x) {
            px += (double)vx[p];
            py += (double)vy[p];
            pz += (double)vz[p];
        }
    }
    m = block_sum(m, sh);
    px = block_sum(px, sh);
    py = block_sum(py, sh);
    pz = block_sum(pz, sh);
    if (threadIdx.x == 0) {
        partial[4 * blockIdx.x + 0] = m;
        partial[4 * blockIdx.x + 1] = px;
        partial[4 * blockIdx.x + 2] = py;
        partial[4 * blockIdx.x + 3] = pz;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_reduce_final(const double* __restrict__ partial, int nblocks,
                                                              double mass, double* __restrict__ out) {
    __shared__ double sh[kRedThreads / 32];
    for (int c = 0; c < 4; ++c) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += partial[4 * b + c];
        v = block_sum(v, sh);
        if (threadIdx.x == 0) out[c] = c == 0 ? v : mass * v;
    }
}

}  // namespace

template <typename T>
int reduce_conserved(Plan& p, const T* mesh, const T* vx, const T* vy, const T* vz, int64_t np, double mass,
                     double* out) {
    const int nblocks = p.num_sms * 4;
    if (!p.red) {
        if (cudaMalloc(&p.red, (size_t)nblocks * 4 * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            p.red = nullptr;
            return fail(PM_ERR_NOMEM, "reduction scratch allocation failed");
        }
        p.bytes += (size_t)nblocks * 4 * sizeof(double);
    }
    double* partial = static_cast<double*>(p.red);
    k_reduce_partials<T><<<nblocks, kRedThreads, 0, p.stream>>>(mesh, p.ng, vx, vy, vz, np, partial);
    k_reduce_final<<<1, kRedThreads, 0, p.stream>>>(partial, nblocks, mass, out);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template int reduce_conserved<float>(Plan&, const float*, const float*, const float*, const float*, int64_t,
                                     double, double*);
template int reduce_conserved<double>(Plan&, const double*, const double*, const double*, const double*,
                                      int64_t, double, double*);

}  // namespace pmb
