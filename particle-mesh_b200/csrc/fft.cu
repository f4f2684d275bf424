// 3D real FFT of the periodic mesh and the Green's-function Poisson solve.
//
// Replaces FFT::forward / FFT::apply_green / FFT::backward of the reference
// (src/fft/fftw/fft.cpp:75-97 over FFTW3-MPI; src/fft/ffte1/fft.cpp:46-68
// over FFTE).  On one GPU there is no slab decomposition and no all-to-all:
// the 3D transform is three passes over HBM, one per axis, each pass a batch
// of 1D transforms held in registers and shared memory.
//
//   z pass  (contiguous): real line of N -> N/2+1 complex via one complex
//           FFT of N/2 and the split-radix real post-processing.
//   y pass  (stride N/2+1) and x pass (stride N (N/2+1)): complex FFTs of
//           N; a block owns TK consecutive kz columns of one plane so every
//           global load / store of a warp is a contiguous run of TK complex.
//   fused x pass: forward x FFT, Green multiply, inverse x FFT in one block,
//           so the Poisson solve costs 5 passes instead of 7.
#include "fft_engine.cuh"

namespace pmb {

template <typename T> constexpr int tk_cols() { return sizeof(T) == 4 ? 16 : 8; }

// ---------------------------------------------------------------- z passes
// Real rows of N (+2 padding) at row stride N+2 reals; as complex a row is
// N/2+1 entries.  LPB rows per block, NTZ threads per row.
template <int N> constexpr int z_threads_per_row() { return threads_per_line<N / 2>(); }
template <int N> constexpr int z_rows_per_block() {
    constexpr int t = z_threads_per_row<N>();
    constexpr int l = 256 / t;
    return l < 1 ? 1 : (l > 64 ? 64 : l);
}

template <typename T, int N>
__global__ void __launch_bounds__(z_threads_per_row<N>() * z_rows_per_block<N>())
k_fft_z_r2c(T* __restrict__ mesh, long long nrows, const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, R1 = Radix<M>::R1, R2 = Radix<M>::R2;
    constexpr int NT = z_threads_per_row<N>(), LPB = z_rows_per_block<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * (M + 1);
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));

    // pass 1 (Ns = 1): global -> registers -> shared
    for (int j = tj; j < M / R1; j += NT) {
        C v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = active ? crow[j + r * (M / R1)] : cmake<C>(0, 0);
        dft<R1, -1>(v);
#pragma unroll
        for (int k = 0; k < R1; ++k) S[j * R1 + k] = v[brev<R1>(k)];
    }
    __syncthreads();
    // pass 2 (Ns = R1): shared -> registers -> shared (natural order)
    C v2[R2];
    const int j2 = tj;
    const bool has2 = j2 < M / R2;
    if (has2) {
#pragma unroll
        for (int r = 0; r < R2; ++r) v2[r] = S[j2 + r * (M / R2)];
#pragma unroll
        for (int r = 1; r < R2; ++r) v2[r] = cmul(v2[r], twiddle<-1>(tw, 2 * r * j2));  // W_M^{r j}
        dft<R2, -1>(v2);
    }
    __syncthreads();
    if (has2) {
#pragma unroll
        for (int k = 0; k < R2; ++k) S[j2 + k * R1] = v2[brev<R2>(k)];
    }
    __syncthreads();
    // real post-processing: X[k] = E[k] + W_N^k O[k], k = 0..M
    if (active) {
        for (int k = tj; k <= M; k += NT) {
            const C zk = S[k == M ? 0 : k];
            const C zc = cconj(S[k == 0 ? 0 : M - k]);
            const C e = cscale(cadd(zk, zc), (T)0.5);
            const C d = csub(zk, zc);
            const C o = cmake<C>((T)0.5 * d.y, (T)-0.5 * d.x);  // -i d / 2
            crow[k] = cadd(e, cmul(twiddle<-1>(tw, k), o));
        }
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(z_threads_per_row<N>() * z_rows_per_block<N>())
k_fft_z_c2r(T* __restrict__ mesh, long long nrows, const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, R1 = Radix<M>::R1, R2 = Radix<M>::R2;
    constexpr int NT = z_threads_per_row<N>(), LPB = z_rows_per_block<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * (M + 1);
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));

    for (int k = tj; k <= M; k += NT) {
        C x = active ? crow[k] : cmake<C>(0, 0);
        if (k == 0 || k == M) x.y = 0;  // FFTW c2r ignores these imaginary parts
        S[k] = x;
    }
    __syncthreads();
    // pre-processing + pass 1: Z[k] = (a + b) + i (a - b) W_N^{-k}, a = X[k], b = conj(X[M-k])
    C v[R1];
    const int j1 = tj;
    const bool has1 = j1 < M / R1;
    if (has1) {
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = j1 + r * (M / R1);
            const C a = S[k], b = cconj(S[M - k]);
            const C s = cadd(a, b), d = cmul(csub(a, b), twiddle<+1>(tw, k));
            v[r] = cmake<C>(s.x - d.y, s.y + d.x);
        }
        dft<R1, +1>(v);
    }
    __syncthreads();
    if (has1) {
#pragma unroll
        for (int k = 0; k < R1; ++k) S[j1 * R1 + k] = v[brev<R1>(k)];
    }
    __syncthreads();
    for (int j = tj; j < M / R2; j += NT) {
        C w[R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) w[r] = S[j + r * (M / R2)];
#pragma unroll
        for (int r = 1; r < R2; ++r) w[r] = cmul(w[r], twiddle<+1>(tw, 2 * r * j));
        dft<R2, +1>(w);
        if (active) {
#pragma unroll
            for (int k = 0; k < R2; ++k) crow[j + k * R1] = w[brev<R2>(k)];
        }
    }
    if (active && tj == 0) crow[M] = cmake<C>(0, 0);  // padding
}

// ------------------------------------------------------ strided C2C passes
// Lines of N complex at element stride `es`; block (bx, by) owns columns
// [bx*TK, bx*TK+TK) of plane `by` (plane base = by * os).
template <typename T, int N>
constexpr int strided_threads() { return tk_cols<T>() * threads_per_line<N>(); }

template <typename T, int N, int DIR>
__global__ void __launch_bounds__(strided_threads<T, N>())
k_fft_strided(typename Cx<T>::t* __restrict__ data, long long es, long long os, int ncols,
              const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int R1 = Radix<N>::R1, R2 = Radix<N>::R2, TK = tk_cols<T>(), NT = threads_per_line<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    C* base = data + (long long)blockIdx.y * os + (active ? col : 0);

    for (int j = ty; j < N / R1; j += NT) {
        C v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = active ? base[(long long)(j + r * (N / R1)) * es] : cmake<C>(0, 0);
        dft<R1, DIR>(v);
#pragma unroll
        for (int k = 0; k < R1; ++k) S[(j * R1 + k) * TK + tx] = v[brev<R1>(k)];
    }
    __syncthreads();
    for (int j = ty; j < N / R2; j += NT) {
        C v[R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) v[r] = S[(j + r * (N / R2)) * TK + tx];
#pragma unroll
        for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], twiddle<DIR>(tw, r * j));
        dft<R2, DIR>(v);
        if (active) {
#pragma unroll
            for (int k = 0; k < R2; ++k) base[(long long)(j + k * R1) * es] = v[brev<R2>(k)];
        }
    }
}

// Green's function G(kx, ky, kz) / N^3 times c (cg = c / N^3).
//   discrete (reference, src/fft/fftw/fft.cpp:55): -cg / (2 (3 - cos - cos - cos));
//     FP64 evaluates exactly that expression from the rounded cosines; FP32
//     uses 3 - sum cos = sum 2 sin^2(pi k/N) to avoid cancellation.
//   spectral: -cg / |k|^2, k = 2 pi m / N with m the signed frequency.
template <typename T>
__device__ __forceinline__ T green_value(int kx, int ky, int kz, int n, int kind, double cg,
                                         const typename Cx<T>::t* __restrict__ tw,
                                         const T* __restrict__ lap1d) {
    if ((kx | ky | kz) == 0) return (T)0;
    if (kind == PM_GREEN_DISCRETE) {
        if constexpr (sizeof(T) == 8) {
            const double s = ((3.0 - (double)__ldg(&tw[kx].x)) - (double)__ldg(&tw[ky].x)) - (double)__ldg(&tw[kz].x);
            return (T)(-cg / (2.0 * s));
        } else {
            const T s = __ldg(lap1d + kx) + __ldg(lap1d + ky) + __ldg(lap1d + kz);
            return (T)(-cg) / ((T)2 * s);
        }
    }
    const int mx = kx <= n / 2 ? kx : kx - n, my = ky <= n / 2 ? ky : ky - n;
    const double w = 6.283185307179586476925286766559 / n;
    const double k2 = w * w * (double)(mx * mx + my * my + kz * kz);
    return (T)(-cg / k2);
}

// Fused x pass of the Poisson solve: forward FFT along x, multiply by G, and
// inverse FFT along x, for TK kz columns of one ky plane.
template <typename T, int N>
__global__ void __launch_bounds__(strided_threads<T, N>())
k_fft_x_green(typename Cx<T>::t* __restrict__ data, long long es, long long os, int ncols,
              const typename Cx<T>::t* __restrict__ tw, const T* __restrict__ lap1d, double cg, int kind) {
    using C = typename Cx<T>::t;
    constexpr int R1 = Radix<N>::R1, R2 = Radix<N>::R2, TK = tk_cols<T>(), NT = threads_per_line<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    const int ky = blockIdx.y;
    C* base = data + (long long)ky * os + (active ? col : 0);

    // forward pass 1: global -> shared
    for (int j = ty; j < N / R1; j += NT) {
        C v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = active ? base[(long long)(j + r * (N / R1)) * es] : cmake<C>(0, 0);
        dft<R1, -1>(v);
#pragma unroll
        for (int k = 0; k < R1; ++k) S[(j * R1 + k) * TK + tx] = v[brev<R1>(k)];
    }
    __syncthreads();
    // forward pass 2 + Green, back into shared (natural kx order)
    {
        C v[R2];
        const int j = ty;
        const bool has = j < N / R2;
        if (has) {
#pragma unroll
            for (int r = 0; r < R2; ++r) v[r] = S[(j + r * (N / R2)) * TK + tx];
#pragma unroll
            for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], twiddle<-1>(tw, r * j));
            dft<R2, -1>(v);
        }
        __syncthreads();
        if (has) {
#pragma unroll
            for (int k = 0; k < R2; ++k) {
                const int kx = j + k * R1;
                const T g = active ? green_value<T>(kx, ky, col, N, kind, cg, tw, lap1d) : (T)0;
                S[kx * TK + tx] = cscale(v[brev<R2>(k)], g);
            }
        }
    }
    __syncthreads();
    // inverse pass 1: shared -> shared
    {
        C v[R1];
        const int j = ty;
        const bool has = j < N / R1;
        if (has) {
#pragma unroll
            for (int r = 0; r < R1; ++r) v[r] = S[(j + r * (N / R1)) * TK + tx];
            dft<R1, +1>(v);
        }
        __syncthreads();
        if (has) {
#pragma unroll
            for (int k = 0; k < R1; ++k) S[(j * R1 + k) * TK + tx] = v[brev<R1>(k)];
        }
    }
    __syncthreads();
    // inverse pass 2: shared -> global
    for (int j = ty; j < N / R2; j += NT) {
        C v[R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) v[r] = S[(j + r * (N / R2)) * TK + tx];
#pragma unroll
        for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], twiddle<+1>(tw, r * j));
        dft<R2, +1>(v);
        if (active) {
#pragma unroll
            for (int k = 0; k < R2; ++k) base[(long long)(j + k * R1) * es] = v[brev<R2>(k)];
        }
    }
}

// Separate Green multiply over the spectrum [kx][ky][kz] (the plain path).
template <typename T>
__global__ void k_green(typename Cx<T>::t* __restrict__ spec, int n, const typename Cx<T>::t* __restrict__ tw,
                        const T* __restrict__ lap1d, double cg, int kind) {
    using C = typename Cx<T>::t;
    const int h = n / 2 + 1;
    const long long total = (long long)n * n * h;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(i % h);
        const long long r = i / h;
        const int ky = (int)(r % n), kx = (int)(r / n);
        const T g = green_value<T>(kx, ky, kz, n, kind, cg, tw, lap1d);
        C v = spec[i];
        spec[i] = cscale(v, g);
    }
}

// ------------------------------------------------------------- launchers
template <typename T, int N> struct Launch {
    using C = typename Cx<T>::t;
    static constexpr int H = N / 2 + 1;
    static size_t smem_z() { return (size_t)z_rows_per_block<N>() * (N / 2 + 1) * sizeof(C); }
    static size_t smem_s() { return (size_t)N * tk_cols<T>() * sizeof(C); }
    static int prepare() {
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_z_r2c<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_z_c2r<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_x_green<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        return PM_OK;
    }
    static void z(const Plan& p, T* mesh, bool forward) {
        const long long rows = (long long)N * N;
        const unsigned grid = (unsigned)((rows + z_rows_per_block<N>() - 1) / z_rows_per_block<N>());
        const int thr = z_threads_per_row<N>() * z_rows_per_block<N>();
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, forward ? ST_FFT_Z_R2C : ST_FFT_Z_C2R);
        if (forward)
            k_fft_z_r2c<T, N><<<grid, thr, smem_z(), p.stream>>>(mesh, rows, tw);
        else
            k_fft_z_c2r<T, N><<<grid, thr, smem_z(), p.stream>>>(mesh, rows, tw);
    }
    // axis 1 = y (stride H, planes x), axis 0 = x (stride N H, planes y)
    static void strided(const Plan& p, T* mesh, int axis, int dir) {
        C* d = reinterpret_cast<C*>(mesh);
        const long long es = axis == 1 ? H : (long long)N * H, os = axis == 1 ? (long long)N * H : H;
        dim3 grid((H + tk_cols<T>() - 1) / tk_cols<T>(), N);
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, axis == 1 ? (dir < 0 ? ST_FFT_Y_FWD : ST_FFT_Y_INV) : (dir < 0 ? ST_FFT_X_FWD : ST_FFT_X_INV));
        if (dir < 0)
            k_fft_strided<T, N, -1><<<grid, strided_threads<T, N>(), smem_s(), p.stream>>>(d, es, os, H, tw);
        else
            k_fft_strided<T, N, +1><<<grid, strided_threads<T, N>(), smem_s(), p.stream>>>(d, es, os, H, tw);
    }
    static void xgreen(const Plan& p, T* mesh, double cg) {
        C* d = reinterpret_cast<C*>(mesh);
        dim3 grid((H + tk_cols<T>() - 1) / tk_cols<T>(), N);
        Timed t(p, ST_FFT_X_GREEN);
        k_fft_x_green<T, N><<<grid, strided_threads<T, N>(), smem_s(), p.stream>>>(
            d, (long long)N * H, H, H, static_cast<const C*>(p.tw), static_cast<const T*>(p.lap1d), cg, p.green_kind);
    }
};

#define PMB_FFT_DISPATCH(NG, ...)                                    \
    switch (NG) {                                                    \
        case 8: { constexpr int N_ = 8; __VA_ARGS__; } break;        \
        case 16: { constexpr int N_ = 16; __VA_ARGS__; } break;      \
        case 32: { constexpr int N_ = 32; __VA_ARGS__; } break;      \
        case 64: { constexpr int N_ = 64; __VA_ARGS__; } break;      \
        case 128: { constexpr int N_ = 128; __VA_ARGS__; } break;    \
        case 256: { constexpr int N_ = 256; __VA_ARGS__; } break;    \
        case 512: { constexpr int N_ = 512; __VA_ARGS__; } break;    \
        case 1024: { constexpr int N_ = 1024; __VA_ARGS__; } break;  \
        default: return fail(PM_ERR_SIZE, "mesh size not supported"); \
    }

bool fft_size_supported(int ng) {
    return ng >= 8 && ng <= 1024 && (ng & (ng - 1)) == 0;
}

int fft_prepare(const Plan& p) {
    int rc = PM_OK;
    if (p.precision == PM_FP64) {
        PMB_FFT_DISPATCH(p.ng, rc = Launch<double, N_>::prepare());
    } else {
        PMB_FFT_DISPATCH(p.ng, rc = Launch<float, N_>::prepare());
    }
    return rc;
}

template <typename T> int fft_r2c(const Plan& p, T* mesh) {
    PMB_FFT_DISPATCH(p.ng, {
        Launch<T, N_>::z(p, mesh, true);
        Launch<T, N_>::strided(p, mesh, 1, -1);
        Launch<T, N_>::strided(p, mesh, 0, -1);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template <typename T> int fft_c2r(const Plan& p, T* mesh) {
    PMB_FFT_DISPATCH(p.ng, {
        Launch<T, N_>::strided(p, mesh, 0, +1);
        Launch<T, N_>::strided(p, mesh, 1, +1);
        Launch<T, N_>::z(p, mesh, false);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

static double green_scale(const Plan& p, double c) {
    const double n = (double)p.ng;
    return c / (n * n * n);
}

template <typename T> int green_apply(const Plan& p, T* mesh, double c_poisson) {
    using C = typename Cx<T>::t;
    const long long total = (long long)p.ng * p.ng * (p.ng / 2 + 1);
    Timed t(p, ST_GREEN);
    k_green<T><<<grid_for(p, total, 256), 256, 0, p.stream>>>(
        reinterpret_cast<C*>(mesh), p.ng, static_cast<const C*>(p.tw), static_cast<const T*>(p.lap1d),
        green_scale(p, c_poisson), p.green_kind);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template <typename T> int poisson_fused(const Plan& p, T* mesh, double c_poisson) {
    const double cg = green_scale(p, c_poisson);
    PMB_FFT_DISPATCH(p.ng, {
        Launch<T, N_>::z(p, mesh, true);
        Launch<T, N_>::strided(p, mesh, 1, -1);
        Launch<T, N_>::xgreen(p, mesh, cg);
        Launch<T, N_>::strided(p, mesh, 1, +1);
        Launch<T, N_>::z(p, mesh, false);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template int fft_r2c<float>(const Plan&, float*);
template int fft_r2c<double>(const Plan&, double*);
template int fft_c2r<float>(const Plan&, float*);
template int fft_c2r<double>(const Plan&, double*);
template int green_apply<float>(const Plan&, float*, double);
template int green_apply<double>(const Plan&, double*, double);
template int poisson_fused<float>(const Plan&, float*, double);
template int poisson_fused<double>(const Plan&, double*, double);

}  // namespace pmb
