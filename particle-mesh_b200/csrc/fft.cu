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
#include <type_traits>

#include "fft_generic.cuh"

namespace pmb {

// Columns per block of the strided passes.  Each warp phase (128 B of
// shared memory) covers whole rows; at N = 1024 (and FP64 N = 512) the tile
// is narrowed so two blocks share an SM and one block's loads overlap the
// other's arithmetic.
template <typename T, int N> constexpr int tk_cols() {
    return sizeof(T) == 4 ? (N >= 1024 ? 8 : 16) : (N >= 1024 ? 4 : 8);
}

// Shared-memory index padding.  z passes: one pad entry after every R1
// entries, so the pass-1 writes j*R1 + k of consecutive j hit distinct
// banks.  Strided passes: TK pad entries after every R1 rows, so the rows
// j*R1 + k of the neighbouring j that share a warp phase differ in bank.
template <int R1, int TK> __device__ __forceinline__ int spad(int row, int tx) {
    return row * TK + tx + TK * (row / R1);
}
// The same padded positions written as base + compile-time offset, for the
// three access patterns of the two-pass schedule (L = R1 R2, R2 % R1 == 0):
//   pass-1 input  j + r R2      pass-1 output  j R1 + k
//   pass-2 input  j + r R1      pass-2 output  j + k R1       (j < R1)
template <int R1, int R2, int TK> struct SIdx {  // strided passes, row stride TK, pad TK per R1 rows
    static __device__ __forceinline__ int in1(int j, int r, int tx) {
        return (j + j / R1) * TK + tx + r * (R2 + R2 / R1) * TK;
    }
    static __device__ __forceinline__ int out1(int j, int k, int tx) { return j * (R1 + 1) * TK + tx + k * TK; }
    static __device__ __forceinline__ int p2(int j, int r, int tx) { return j * TK + tx + r * (R1 + 1) * TK; }
};

// ---------------------------------------------------------------- z passes
// Real rows of N (+2 padding) at a row stride of N+2 reals; as complex a row
// is M+1 = N/2+1 entries.  NT threads per row, LPB rows per block.
template <int N> constexpr int z_threads_per_row() { return threads_per_line<N / 2>(); }
// Small blocks (64 threads: 4 rows of 1024 in FP32) let many independent
// blocks per SM interleave their load and compute phases; the FP64 R2C runs
// best with 128 (measured on B200).
template <typename T, int N, bool C2R> constexpr int z_rows_per_block() {
    constexpr int thr = (sizeof(T) == 4 || C2R) ? 64 : 128;
    constexpr int l = thr / z_threads_per_row<N>();
    return l < 1 ? 1 : (l > 64 ? 64 : l);
}
template <typename T, int N, bool C2R> constexpr int z_threads() {
    return z_threads_per_row<N>() * z_rows_per_block<T, N, C2R>();
}

// R2C along z: complex FFT of the M packed pairs (x[2n], x[2n+1]), then
// X[k] = E[k] + W_N^k O[k], E = (Z[k] + conj Z[M-k]) / 2, O = -i (Z[k] - conj Z[M-k]) / 2.
template <typename T, int N>
__global__ void __launch_bounds__(z_threads<T, N, false>(), 2)
k_fft_z_r2c(T* __restrict__ mesh, long long nrows, const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, R1 = Radix<M>::R1, R2 = Radix<M>::R2;
    constexpr int NT = z_threads_per_row<N>(), LPB = z_rows_per_block<T, N, false>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * z_row_stride<N>();
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));

    using I = ZIdx<R1, R2>;
    stockham_pass1<R1, R2, -1, false, C>(
        tj, [&](int j, int r) { return active ? crow[j + r * R2] : cmake<C>(0, 0); },
        [&](int j, int k, C v) { S[I::out1(j, k)] = v; });
    __syncthreads();
    // (the register form of the post-processing, r2c_post, measured slower
    // here than this shared-memory one: 5.17 vs 4.13 ms for the FP64 pass at
    // 1024^3, from register spills)
    stockham_pass2<R1, R2, -1, true, C>(
        tj, [&](int j, int r) { return S[I::p2(j, r)]; }, [&](int j, int k, C v) { S[I::p2(j, k)] = v; },
        pass2_twiddles<-1, (R2 >= 16 && sizeof(T) == 4), 2>(tw, tj));
    __syncthreads();
    auto sld = [&](int i) { return S[zpad<R1>(i)]; };
    if (active) {
        for (int k = tj; k <= M; k += NT) {
            const C zk = sld(k == M ? 0 : k);
            const C zc = cconj(sld(k == 0 ? 0 : M - k));
            const C e = cscale(cadd(zk, zc), (T)0.5);
            const C d = csub(zk, zc);
            const C o = cmake<C>((T)0.5 * d.y, (T)-0.5 * d.x);  // -i d / 2
            crow[k] = cadd(e, cmul(twiddle<-1>(tw, k), o));
        }
    }
}

// C2R along z: Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) W_N^-k,
// inverse complex FFT of M, unpacked to reals.  The imaginary parts of X[0]
// and X[M] are ignored (FFTW c2r semantics); the row padding is zeroed.
template <typename T, int N>
__global__ void __launch_bounds__(z_threads<T, N, true>(), 2)
k_fft_z_c2r(T* __restrict__ mesh, long long nrows, const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, R1 = Radix<M>::R1, R2 = Radix<M>::R2;
    constexpr int NT = z_threads_per_row<N>(), LPB = z_rows_per_block<T, N, true>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * z_row_stride<N>();
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));

    // the pre-processing pairs X[k] with X[M - k]: both are read from global
    // memory (the second read of each element hits L1) straight into pass 1,
    // so no shared-memory staging of the row is needed (FP32 at 1024^3: 1.53
    // vs 1.60 ms; FP64: 3.62 vs 3.76 ms)
    auto gld = [&](int k) {
        C v = active ? crow[k] : cmake<C>(0, 0);
        if (k == 0 || k == M) v.y = 0;
        return v;
    };
    using I = ZIdx<R1, R2>;
    auto pre = [&](int j, int r) {
        const int k = j + r * R2;
        const C a = gld(k), b = cconj(gld(M - k));
        const C s = cadd(a, b), d = cmul(csub(a, b), twiddle<+1>(tw, k));
        return cmake<C>(s.x - d.y, s.y + d.x);
    };
    stockham_pass1<R1, R2, +1, false, C>(tj, pre, [&](int j, int k, C v) { S[I::out1(j, k)] = v; });
    __syncthreads();
    stockham_pass2<R1, R2, +1, false, C>(
        tj, [&](int j, int r) { return S[I::p2(j, r)]; },
        [&](int j, int k, C v) { if (active) crow[j + k * R1] = v; },
        pass2_twiddles<+1, (R2 >= 16 && sizeof(T) == 4), 2>(tw, tj));
    if (active && tj == 0) crow[M] = cmake<C>(0, 0);  // padding
}

// ------------------------------------------------------ strided C2C passes
// Lines of N complex at element stride `es`; block (bx, by) owns columns
// [bx*TK, bx*TK+TK) of plane `by` (plane base = by * os).
template <int N, int TK, int RV = 0> constexpr int strided_threads() { return TK * threads_per_line_v<N, RV>(); }
template <int N, int TK, int RV = 0> constexpr int strided_smem_elems() { return (N + N / RadixV<N, RV>::R1) * TK; }

template <typename T, int N, int DIR, int TK, int RV = 0, int AX = -1>
__global__ void __launch_bounds__(strided_threads<N, TK, RV>(), 2)
k_fft_strided(typename Cx<T>::t* __restrict__ data, long long es_, long long os_, long long bs, int ncols,
              const typename Cx<T>::t* __restrict__ tw, typename Cx<T>::t* out, PeerMap po = PeerMap{}) {
    using C = typename Cx<T>::t;
    constexpr int R1 = RadixV<N, RV>::R1, R2 = RadixV<N, RV>::R2;
    // AX = 1 (y) or 0 (x): the element and plane strides of the padded
    // spectrum are compile-time constants, so the 2 R2 accesses of a thread
    // are one base address plus constant offsets; AX = -1 takes them as given.
    // AX = 2: lines read along the outer axis of `data` (element stride N H,
    // plane stride H: y lines of the transposed spectrum [ky][kx][kz]) and
    // written along the middle axis of `out` (element stride H, plane stride
    // N H: the spectrum [kx][y][kz]).
    // AX = 3: y lines of the planes [x][y][kz] of `data` written into `out`
    // at the runtime strides es_ (element) and os_ (plane): the x-slab's y
    // forward pass storing straight into its transpose buffer.
    // AX = 4: lines read from `data` at the runtime strides es_, os_ and
    // written along the middle axis of `out` (stride H, planes N H): the
    // x-slab's y inverse pass reading straight from its transpose buffer.
    // AX = 5: y lines of the planes [x][y][kz] of `data` stored through the
    // peer map `po` (the x-slab's y forward into the owners' buffers).
    // AX = 0, 1, -1 work in place.
    constexpr long long H = N / 2 + 1;
    constexpr bool OUTER = AX == 0 || AX == 2;
    constexpr bool MID_IN = AX == 1 || AX == 3 || AX == 5, MID_OUT = AX == 2 || AX == 4;
    const long long es = MID_IN ? H : (OUTER ? (long long)N * H : es_);
    const long long os = MID_IN ? (long long)N * H : (OUTER ? H : os_);
    const long long oes = MID_OUT ? H : (AX == 3 ? es_ : es), oos = MID_OUT ? (long long)N * H : (AX == 3 ? os_ : os);
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    // plane blockIdx.y % N of box blockIdx.y / N (boxes of a batch at stride bs)
    const long long box = blockIdx.y / N, plane = blockIdx.y % N;
    C* base = data + box * bs + plane * os + (active ? col : 0);
    C* obase = AX >= 2 ? out + box * bs + plane * oos + (active ? col : 0) : base;

    using I = SIdx<R1, R2, TK>;
    const long long es1 = es * R2, oes2 = oes * R1;
    stockham_pass1<R1, R2, DIR, false, C>(
        ty, [&](int j, int r) { return active ? base[j * es + r * es1] : cmake<C>(0, 0); },
        [&](int j, int k, C v) { S[I::out1(j, k, tx)] = v; });
    __syncthreads();
    stockham_pass2<R1, R2, DIR, false, C>(
        ty, [&](int j, int r) { return S[I::p2(j, r, tx)]; },
        [&](int j, int k, C v) {
            if (!active) return;
            if constexpr (AX == 5) {
                const int m = j + k * R1;
                reinterpret_cast<C*>(po.base[m >> po.sl])[(long long)plane * po.ps + (m & po.mask) * po.s0 + col] = v;
            } else {
                obase[j * oes + k * oes2] = v;
            }
        },
        pass2_twiddles<DIR, (R2 >= 16 && sizeof(T) == 4)>(tw, ty));
}

// Lines of N complex read from `in` and written to `out` through line maps
// (plane blockIdx.y, columns [bx TK, bx TK + TK) consecutive): the y passes
// of a pencil, reading the blocks one transpose delivered and writing the
// blocks the next one sends.
// PEER: the outputs go through the peer map `po` instead of `out` / `mo`.
template <typename T, int N, int DIR, int TK, int RV = 0, bool PEER = false>
__global__ void __launch_bounds__(strided_threads<N, TK, RV>(), 2)
k_fft_lines_map(const typename Cx<T>::t* __restrict__ in, typename Cx<T>::t* __restrict__ out, LineMap mi,
                LineMap mo, int ncols, const typename Cx<T>::t* __restrict__ tw, PeerMap po = PeerMap{}) {
    using C = typename Cx<T>::t;
    constexpr int R1 = RadixV<N, RV>::R1, R2 = RadixV<N, RV>::R2;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    const C* ib = in + (long long)blockIdx.y * mi.ps + (active ? col : 0);
    C* ob = out + (long long)blockIdx.y * mo.ps + (active ? col : 0);
    using I = SIdx<R1, R2, TK>;
    stockham_pass1<R1, R2, DIR, false, C>(
        ty, [&](int j, int r) { return active ? ib[lm_off(mi, j + r * R2)] : cmake<C>(0, 0); },
        [&](int j, int k, C v) { S[I::out1(j, k, tx)] = v; });
    __syncthreads();
    stockham_pass2<R1, R2, DIR, false, C>(
        ty, [&](int j, int r) { return S[I::p2(j, r, tx)]; },
        [&](int j, int k, C v) {
            if (!active) return;
            const int m = j + k * R1;
            if (PEER)
                reinterpret_cast<C*>(po.base[m >> po.sl])[(long long)blockIdx.y * po.ps + (m & po.mask) * po.s0 + col] = v;
            else
                ob[lm_off(mo, m)] = v;
        },
        pass2_twiddles<DIR, (R2 >= 16 && sizeof(T) == 4)>(tw, ty));
}

// Green's function times c / N^3 (cg = c / N^3) at (kx, ky, kz).
//   FP64 discrete: -cg / (2 (3 - cos - cos - cos)), the reference's own
//     expression (src/fft/fftw/fft.cpp:55) on the rounded cosines.
//   otherwise: -cg / (g1d[kx] + g1d[ky] + g1d[kz]) with the plan's 1D table
//     g1d = 4 sin^2(pi k/N) (discrete: 2 (3 - sum cos) without cancellation)
//     or (2 pi m/N)^2, m the signed frequency (spectral).
template <typename T>
__device__ __forceinline__ T green_value(int kx, int ky, int kz, int kind, double cg,
                                         const typename Cx<T>::t* __restrict__ tw,
                                         const T* __restrict__ g1d) {
    if ((kx | ky | kz) == 0) return (T)0;
    if constexpr (sizeof(T) == 8) {
        if (kind == PM_GREEN_DISCRETE) {
            const double s = ((3.0 - (double)__ldg(&tw[kx].x)) - (double)__ldg(&tw[ky].x)) - (double)__ldg(&tw[kz].x);
            return (T)(-cg / (2.0 * s));
        }
        return (T)(-cg / ((double)__ldg(g1d + kx) + (double)__ldg(g1d + ky) + (double)__ldg(g1d + kz)));
    } else {
        const float s = __ldg(g1d + kx) + __ldg(g1d + ky) + __ldg(g1d + kz);
        // fast division (2 ulp): the correctly rounded reciprocal cost a
        // sixth of the x + Green pass
        return __fdividef((float)(-cg), s);
    }
}

// green_value along one x line (fixed ky, kz): the line's two table entries
// loaded once, every element summed in green_value's order (same results).
template <typename T> struct GreenLine {
    using C = typename Cx<T>::t;
    int ky, kz, kind;
    double cg;
    const C* __restrict__ tw;
    const T* __restrict__ g1d;
    T gy = 0, gz = 0;
    __device__ __forceinline__ GreenLine(int ky_, int kz_, int kind_, double cg_, const C* __restrict__ tw_,
                                         const T* __restrict__ g1d_, bool active)
        : ky(ky_), kz(kz_), kind(kind_), cg(cg_), tw(tw_), g1d(g1d_) {
        if (!active) return;
        if (sizeof(T) == 8 && kind == PM_GREEN_DISCRETE) {
            gy = (T)__ldg(&tw[ky].x);
            gz = (T)__ldg(&tw[kz].x);
        } else {
            gy = __ldg(g1d + ky);
            gz = __ldg(g1d + kz);
        }
    }
    __device__ __forceinline__ T operator()(int kx) const {
        if ((kx | ky | kz) == 0) return (T)0;
        if constexpr (sizeof(T) == 8) {
            if (kind == PM_GREEN_DISCRETE) {
                const double s = ((3.0 - (double)__ldg(&tw[kx].x)) - (double)gy) - (double)gz;
                return (T)(-cg / (2.0 * s));
            }
            return (T)(-cg / (((double)__ldg(g1d + kx) + (double)gy) + (double)gz));
        } else {
            return __fdividef((float)(-cg), (__ldg(g1d + kx) + gy) + gz);
        }
    }
};

// Fused x pass of the Poisson solve: forward FFT along x, multiply by G,
// inverse FFT along x, for TK kz columns of one ky plane.  XT: the lines are
// written to `out` in the transposed layout [ky][kx][kz] (element stride H),
// so that neither this pass nor the next one both reads and writes lines
// whose elements lie N H apart; otherwise in place.
// SLABX: the x lines of a decomposed mesh's share of the spectrum, read
// from the received transpose buffer `data` and written to the one to send
// back, `out`, both through the line map `lm` (plane blockIdx.y holds
// ky = ky0 + blockIdx.y, column c holds kz = kz0 + c).  An x-slab's blocks
// [rank][kyl][x][kz] map kx to (kx >> log2 nx) nx^2 H + (kx & (nx - 1)) H; a
// pencil's [kx][kyl][kz] to kx yc hc.
// PEER (with SLABX): the outputs go through the peer map `po` (element kx to
// the rank owning x = kx) instead of `out`.
template <typename T, int N, int TK, int RV = 0, bool XT = false, bool SLABX = false, bool PEER = false>
__global__ void __launch_bounds__(strided_threads<N, TK, RV>(), 2)
k_fft_x_green(typename Cx<T>::t* __restrict__ data, long long es_, long long os_, long long bs, int ncols,
              const typename Cx<T>::t* __restrict__ tw, const T* __restrict__ g1d, double cg, int kind,
              typename Cx<T>::t* out, int ky0 = 0, LineMap lm = LineMap{}, int kz0 = 0, PeerMap po = PeerMap{}) {
    using C = typename Cx<T>::t;
    constexpr int R1 = RadixV<N, RV>::R1, R2 = RadixV<N, RV>::R2;
    // x lines of the padded spectrum: compile-time strides (es_ = N H and
    // os_ = H are what every caller passes)
    constexpr long long es = (long long)N * (N / 2 + 1), os = N / 2 + 1;
    constexpr long long oes = XT ? os : es, oos = XT ? es : os;
    // FP32: pass-2 twiddles from 10 table loads per thread (2.97 vs 3.10 ms)
    constexpr bool kSplitTw = R2 >= 16 && sizeof(T) == 4;
    (void)es_;
    (void)os_;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* S = reinterpret_cast<C*>(smraw);
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    const int ky = SLABX ? ky0 + (int)blockIdx.y : (int)(blockIdx.y % N);
    auto soff = [&](int n) { return lm_off(lm, n); };
    C* base = SLABX ? data + (long long)blockIdx.y * lm.ps + (active ? col : 0)
                    : data + (long long)(blockIdx.y / N) * bs + (long long)ky * os + (active ? col : 0);
    C* obase = SLABX ? out + (long long)blockIdx.y * lm.ps + (active ? col : 0)
                     : (XT ? out + (long long)(blockIdx.y / N) * bs + (long long)ky * oos + (active ? col : 0) : base);

    using I = SIdx<R1, R2, TK>;
    const long long es1 = es * R2, oes2 = oes * R1;
    auto p2ld = [&](int j, int r) { return S[I::p2(j, r, tx)]; };
    stockham_pass1<R1, R2, -1, false, C>(
        ty,
        [&](int j, int r) {
            if (!active) return cmake<C>(0, 0);
            return SLABX ? base[soff(j + r * R2)] : base[j * es + r * es1];
        },
        [&](int j, int k, C v) { S[I::out1(j, k, tx)] = v; });
    __syncthreads();
    const GreenLine<T> green(ky, col + kz0, kind, cg, tw, g1d, active);
    stockham_pass2<R1, R2, -1, true, C>(
        ty, p2ld,
        [&](int j, int k, C v) { S[I::p2(j, k, tx)] = cscale(v, active ? green(j + k * R1) : (T)0); },
        pass2_twiddles<-1, kSplitTw>(tw, ty));
    __syncthreads();
    stockham_pass1<R1, R2, +1, true, C>(
        ty, [&](int j, int r) { return S[I::in1(j, r, tx)]; }, [&](int j, int k, C v) { S[I::out1(j, k, tx)] = v; });
    __syncthreads();
    stockham_pass2<R1, R2, +1, false, C>(
        ty, p2ld,
        [&](int j, int k, C v) {
            if (!active) return;
            if (PEER) {
                const int m = j + k * R1;
                reinterpret_cast<C*>(po.base[m >> po.sl])[(long long)blockIdx.y * po.ps + (m & po.mask) * po.s0 + col] = v;
            } else if (SLABX) {
                obase[soff(j + k * R1)] = v;
            } else {
                obase[j * oes + k * oes2] = v;
            }
        },
        pass2_twiddles<+1, kSplitTw>(tw, ty));
}

// Separate Green multiply over the spectrum [kx][ky][kz] (the plain path):
// one block iteration per (kx, ky) row, threads along kz.
template <typename T>
__global__ void k_green(typename Cx<T>::t* __restrict__ spec, int n, const typename Cx<T>::t* __restrict__ tw,
                        const T* __restrict__ g1d, double cg, int kind) {
    const int h = n / 2 + 1;
    for (long long row = blockIdx.x; row < (long long)n * n; row += gridDim.x) {
        const int kx = (int)(row / n), ky = (int)(row % n);
        typename Cx<T>::t* r = spec + row * h;
        for (int kz = threadIdx.x; kz < h; kz += blockDim.x)
            r[kz] = cscale(r[kz], green_value<T>(kx, ky, kz, kind, cg, tw, g1d));
    }
}

// ------------------------------- mixed-radix sizes (2^a 3^b 5^c): generic passes
template <int N> constexpr int g_z_rows() { return 256 / GRadix<N / 2>::NT; }
// Columns per block of the generic strided passes: the widest of 16, 8, 4, 2
// whose two ping-pong line buffers fit 96 KB (two blocks per SM).
template <typename T, int N> constexpr int gtk() {
    constexpr size_t c = 2 * sizeof(T);
    return 2 * (size_t)N * 16 * c <= 98304 ? 16 : (2 * (size_t)N * 8 * c <= 98304 ? 8 : (2 * (size_t)N * 4 * c <= 98304 ? 4 : 2));
}

template <typename T, int N>
__global__ void __launch_bounds__(256) k_fftg_z_r2c(T* __restrict__ mesh, long long nrows,
                                                    const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, NT = GRadix<M>::NT, LPB = g_z_rows<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * 2 * (M + 1);
    C* B = A + (M + 1);
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));
    for (int k = tj; k < M; k += NT) A[k] = active ? crow[k] : cmake<C>(0, 0);
    __syncthreads();
    const C* Z = gfft<M, -1>(A, B, tj, [](int e) { return e; }, tw, 2);
    if (active) {
        for (int k = tj; k <= M; k += NT) {
            const C zk = Z[k == M ? 0 : k];
            const C zc = cconj(Z[k == 0 ? 0 : M - k]);
            const C e = cscale(cadd(zk, zc), (T)0.5);
            const C d = csub(zk, zc);
            const C o = cmake<C>((T)0.5 * d.y, (T)-0.5 * d.x);
            crow[k] = cadd(e, cmul(twiddle<-1>(tw, k), o));
        }
    }
}

template <typename T, int N>
__global__ void __launch_bounds__(256) k_fftg_z_c2r(T* __restrict__ mesh, long long nrows,
                                                    const typename Cx<T>::t* __restrict__ tw) {
    using C = typename Cx<T>::t;
    constexpr int M = N / 2, NT = GRadix<M>::NT, LPB = g_z_rows<N>();
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw) + (threadIdx.x / NT) * 2 * (M + 1);
    C* B = A + (M + 1);
    const int tj = threadIdx.x % NT;
    const long long row = (long long)blockIdx.x * LPB + threadIdx.x / NT;
    const bool active = row < nrows;
    C* crow = reinterpret_cast<C*>(mesh + (active ? row : 0) * (long long)(N + 2));
    for (int k = tj; k <= M; k += NT) {
        C x = active ? crow[k] : cmake<C>(0, 0);
        if (k == 0 || k == M) x.y = 0;
        A[k] = x;
    }
    __syncthreads();
    for (int k = tj; k < M; k += NT) {
        const C a = A[k], b = cconj(A[M - k]);
        const C s = cadd(a, b), d = cmul(csub(a, b), twiddle<+1>(tw, k));
        B[k] = cmake<C>(s.x - d.y, s.y + d.x);
    }
    __syncthreads();
    const C* z = gfft<M, +1>(B, A, tj, [](int e) { return e; }, tw, 2);
    if (active) {
        for (int k = tj; k < M; k += NT) crow[k] = z[k];
        if (tj == 0) crow[M] = cmake<C>(0, 0);
    }
}

template <typename T, int N, int DIR, bool GREEN, int TK>
__global__ void __launch_bounds__(TK * GRadix<N>::NT)
k_fftg_strided(typename Cx<T>::t* __restrict__ data, long long es, long long os, long long bs, int ncols,
               const typename Cx<T>::t* __restrict__ tw, const T* __restrict__ g1d, double cg, int kind) {
    using C = typename Cx<T>::t;
    constexpr int NT = GRadix<N>::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    C* A = reinterpret_cast<C*>(smraw);
    C* B = A + N * TK;
    const int tx = threadIdx.x % TK, ty = threadIdx.x / TK;
    const int col = blockIdx.x * TK + tx;
    const bool active = col < ncols;
    const int plane = blockIdx.y % N, box = blockIdx.y / N;
    C* base = data + box * bs + plane * os + (active ? col : 0);
    auto ix = [&](int e) { return e * TK + tx; };
    for (int e = ty; e < N; e += NT) A[ix(e)] = active ? base[e * es] : cmake<C>(0, 0);
    __syncthreads();
    C* r = gfft<N, DIR>(A, B, ty, ix, tw, 1);
    if constexpr (GREEN) {
        for (int e = ty; e < N; e += NT)
            r[ix(e)] = cscale(r[ix(e)], active ? green_value<T>(e, plane, col, kind, cg, tw, g1d) : (T)0);
        __syncthreads();
        r = gfft<N, +1>(r, r == A ? B : A, ty, ix, tw, 1);
    }
    if (active)
        for (int e = ty; e < N; e += NT) base[e * es] = r[ix(e)];
}

template <typename T, int N, int TK = gtk<T, N>()> struct LaunchG {
    using C = typename Cx<T>::t;
    static constexpr int H = N / 2 + 1;
    static constexpr bool kTransposedX = false;
    static void xgreen_yinv_transposed(const Plan&, T*, T*, double) {}
    static size_t smem_z() { return (size_t)g_z_rows<N>() * 2 * (N / 2 + 1) * sizeof(C); }
    static size_t smem_s() { return (size_t)2 * N * TK * sizeof(C); }
    static int prepare() {
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fftg_z_r2c<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fftg_z_c2r<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fftg_strided<T, N, -1, false, TK>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fftg_strided<T, N, +1, false, TK>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fftg_strided<T, N, -1, true, TK>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        return PM_OK;
    }
    static void z(const Plan& p, T* mesh, bool forward, int nbox = 1) {
        const long long rows = (long long)nbox * N * N;
        const unsigned grid = (unsigned)((rows + g_z_rows<N>() - 1) / g_z_rows<N>());
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, forward ? ST_FFT_Z_R2C : ST_FFT_Z_C2R);
        if (forward)
            k_fftg_z_r2c<T, N><<<grid, 256, smem_z(), p.stream>>>(mesh, rows, tw);
        else
            k_fftg_z_c2r<T, N><<<grid, 256, smem_z(), p.stream>>>(mesh, rows, tw);
    }
    static void strided(const Plan& p, T* mesh, int axis, int dir, int nbox = 1) {
        C* d = reinterpret_cast<C*>(mesh);
        const long long es = axis == 1 ? H : (long long)N * H, os = axis == 1 ? (long long)N * H : H;
        dim3 grid((H + TK - 1) / TK, N * nbox);
        const C* tw = static_cast<const C*>(p.tw);
        const T* g = static_cast<const T*>(p.g1d);
        Timed t(p, axis == 1 ? (dir < 0 ? ST_FFT_Y_FWD : ST_FFT_Y_INV) : (dir < 0 ? ST_FFT_X_FWD : ST_FFT_X_INV));
        const long long bs = (long long)N * N * H;
        if (dir < 0)
            k_fftg_strided<T, N, -1, false, TK><<<grid, TK * GRadix<N>::NT, smem_s(), p.stream>>>(d, es, os, bs, H, tw, g, 0.0, 0);
        else
            k_fftg_strided<T, N, +1, false, TK><<<grid, TK * GRadix<N>::NT, smem_s(), p.stream>>>(d, es, os, bs, H, tw, g, 0.0, 0);
    }
    static void xgreen(const Plan& p, T* mesh, double cg, int nbox = 1) {
        C* d = reinterpret_cast<C*>(mesh);
        dim3 grid((H + TK - 1) / TK, N * nbox);
        Timed t(p, ST_FFT_X_GREEN);
        k_fftg_strided<T, N, -1, true, TK><<<grid, TK * GRadix<N>::NT, smem_s(), p.stream>>>(
            d, (long long)N * H, H, (long long)N * N * H, H, static_cast<const C*>(p.tw), static_cast<const T*>(p.g1d),
            cg, p.green_kind);
    }
};

// ------------------------------------------------------------- launchers
template <typename T, int N, int TK = tk_cols<T, N>(), int RV = 0> struct Launch {
    using C = typename Cx<T>::t;
    static constexpr int H = N / 2 + 1;
    static size_t smem_z(bool c2r) {
        return (size_t)(c2r ? z_rows_per_block<T, N, true>() : z_rows_per_block<T, N, false>()) * z_row_stride<N>() *
               sizeof(C);
    }
    static size_t smem_s() { return (size_t)strided_smem_elems<N, TK, RV>() * sizeof(C); }
    static int prepare() {
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_z_r2c<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z(false)));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_z_c2r<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_z(true)));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, -1, TK, RV, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, +1, TK, RV, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, -1, TK, RV, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, +1, TK, RV, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_x_green<T, N, TK, RV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_x_green<T, N, TK, RV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, +1, TK, RV, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, -1, TK, RV, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, -1, TK, RV, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_strided<T, N, +1, TK, RV, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_lines_map<T, N, -1, TK, RV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_lines_map<T, N, -1, TK, RV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_lines_map<T, N, +1, TK, RV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_x_green<T, N, TK, RV, false, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_lines_map<T, N, +1, TK, RV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        PMB_CUDA_CHECK(cudaFuncSetAttribute(k_fft_x_green<T, N, TK, RV, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s()));
        return PM_OK;
    }
    // ---- x-slab decomposition: passes over part of a mesh
    // z pass over `rows` rows of N reals (+2 padding)
    static void z_rows(const Plan& p, T* mesh, bool forward, long long rows) {
        const int lpb = forward ? z_rows_per_block<T, N, false>() : z_rows_per_block<T, N, true>();
        const unsigned grid = (unsigned)((rows + lpb - 1) / lpb);
        const int thr = z_threads_per_row<N>() * lpb;
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, forward ? ST_FFT_Z_R2C : ST_FFT_Z_C2R);
        if (forward)
            k_fft_z_r2c<T, N><<<grid, thr, smem_z(false), p.stream>>>(mesh, rows, tw);
        else
            k_fft_z_c2r<T, N><<<grid, thr, smem_z(true), p.stream>>>(mesh, rows, tw);
    }
    // y lines of `planes` consecutive x planes [x][y][kz]
    static void y_planes(const Plan& p, T* mesh, int dir, int planes) {
        C* d = reinterpret_cast<C*>(mesh);
        const dim3 grid((H + TK - 1) / TK, planes);
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, dir < 0 ? ST_FFT_Y_FWD : ST_FFT_Y_INV);
        if (dir < 0)
            k_fft_strided<T, N, -1, TK, RV, 1><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                d, H, (long long)N * H, 0, H, tw, d);
        else
            k_fft_strided<T, N, +1, TK, RV, 1><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                d, H, (long long)N * H, 0, H, tw, d);
    }
    // lines through line maps (pencil y passes)
    static void lines_map(const Plan& p, const T* in, T* out, LineMap mi, LineMap mo, int planes, int ncols, int dir,
                          int stage) {
        const dim3 grid((ncols + TK - 1) / TK, planes);
        const C* tw = static_cast<const C*>(p.tw);
        const C* i = reinterpret_cast<const C*>(in);
        C* o = reinterpret_cast<C*>(out);
        Timed t(p, stage);
        if (dir < 0)
            k_fft_lines_map<T, N, -1, TK, RV><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                i, o, mi, mo, ncols, tw);
        else
            k_fft_lines_map<T, N, +1, TK, RV><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                i, o, mi, mo, ncols, tw);
    }
    // x forward + Green + x inverse of `planes` ky planes (ky0 + plane) and
    // ncols kz columns (kz0 + column) through the line map m, from `in` to `out`
    static void xgreen_map(const Plan& p, const T* in, T* out, double cg, LineMap m, int planes, int ncols, int ky0,
                           int kz0) {
        const dim3 grid((ncols + TK - 1) / TK, planes);
        Timed t(p, ST_FFT_X_GREEN);
        k_fft_x_green<T, N, TK, RV, false, true><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            const_cast<C*>(reinterpret_cast<const C*>(in)), H, (long long)N * H, 0, ncols, static_cast<const C*>(p.tw),
            static_cast<const T*>(p.g1d), cg, p.green_kind, reinterpret_cast<C*>(out), ky0, m, kz0);
    }
    // the y forward of an x-slab's own planes storing each ky row straight
    // into the rank owning ky (peer map), and x + Green likewise by kx
    static void y_to_peers(const Plan& p, const T* own, const PeerMap& po, int nx) {
        const dim3 grid((H + TK - 1) / TK, nx);
        Timed t(p, ST_FFT_Y_FWD);
        k_fft_strided<T, N, -1, TK, RV, 5><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            const_cast<C*>(reinterpret_cast<const C*>(own)), H, (long long)N * H, 0, H, static_cast<const C*>(p.tw),
            nullptr, po);
    }
    static void xgreen_peers(const Plan& p, const T* in, double cg, LineMap m, const PeerMap& po, int planes,
                             int ncols, int ky0, int kz0) {
        const dim3 grid((ncols + TK - 1) / TK, planes);
        Timed t(p, ST_FFT_X_GREEN);
        k_fft_x_green<T, N, TK, RV, false, true, true><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            const_cast<C*>(reinterpret_cast<const C*>(in)), H, (long long)N * H, 0, ncols,
            static_cast<const C*>(p.tw), static_cast<const T*>(p.g1d), cg, p.green_kind, nullptr, ky0, m, kz0, po);
    }
    // lines read through a line map, stored through a peer map (pencil y passes)
    static void lines_peers(const Plan& p, const T* in, LineMap mi, const PeerMap& po, int planes, int ncols, int dir,
                            int stage) {
        const dim3 grid((ncols + TK - 1) / TK, planes);
        const C* tw = static_cast<const C*>(p.tw);
        const C* i = reinterpret_cast<const C*>(in);
        Timed t(p, stage);
        if (dir < 0)
            k_fft_lines_map<T, N, -1, TK, RV, true><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                i, nullptr, mi, LineMap{}, ncols, tw, po);
        else
            k_fft_lines_map<T, N, +1, TK, RV, true><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                i, nullptr, mi, LineMap{}, ncols, tw, po);
    }
    // y forward of the nx own planes [x][y][kz] of an x-slab, stored as the
    // rows [ky][x][kz] of its transpose buffer
    static void y_to_rows(const Plan& p, const T* own, T* rows, int nx) {
        const dim3 grid((H + TK - 1) / TK, nx);
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, ST_FFT_Y_FWD);
        k_fft_strided<T, N, -1, TK, RV, 3><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            const_cast<C*>(reinterpret_cast<const C*>(own)), (long long)nx * H, H, 0, H, tw,
            reinterpret_cast<C*>(rows));
    }
    // y inverse from the rows [ky][x][kz] of an x-slab's transpose buffer
    // into its nx own planes [x][y][kz]
    static void y_from_rows(const Plan& p, const T* rows, T* own, int nx) {
        const dim3 grid((H + TK - 1) / TK, nx);
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, ST_FFT_Y_INV);
        k_fft_strided<T, N, +1, TK, RV, 4><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            const_cast<C*>(reinterpret_cast<const C*>(rows)), (long long)nx * H, H, 0, H, tw,
            reinterpret_cast<C*>(own));
    }
    static constexpr bool kTransposedX = true;
    static void z(const Plan& p, T* mesh, bool forward, int nbox = 1) {
        const long long rows = (long long)nbox * N * N;
        const int lpb = forward ? z_rows_per_block<T, N, false>() : z_rows_per_block<T, N, true>();
        const unsigned grid = (unsigned)((rows + lpb - 1) / lpb);
        const int thr = z_threads_per_row<N>() * lpb;
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, forward ? ST_FFT_Z_R2C : ST_FFT_Z_C2R);
        if (forward)
            k_fft_z_r2c<T, N><<<grid, thr, smem_z(false), p.stream>>>(mesh, rows, tw);
        else
            k_fft_z_c2r<T, N><<<grid, thr, smem_z(true), p.stream>>>(mesh, rows, tw);
    }
    // axis 1 = y (stride H, planes x), axis 0 = x (stride N H, planes y); a
    // batch of nbox meshes lies at a stride of N^2 H complex
    static void strided(const Plan& p, T* mesh, int axis, int dir, int nbox = 1) {
        C* d = reinterpret_cast<C*>(mesh);
        const long long es = axis == 1 ? H : (long long)N * H, os = axis == 1 ? (long long)N * H : H;
        const long long bs = (long long)N * N * H;
        dim3 grid((H + TK - 1) / TK, N * nbox);
        const C* tw = static_cast<const C*>(p.tw);
        Timed t(p, axis == 1 ? (dir < 0 ? ST_FFT_Y_FWD : ST_FFT_Y_INV) : (dir < 0 ? ST_FFT_X_FWD : ST_FFT_X_INV));
        auto go = [&](auto dirc, auto axc) {
            k_fft_strided<T, N, decltype(dirc)::value, TK, RV, decltype(axc)::value>
                <<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(d, es, os, bs, H, tw, d);
        };
        using F = std::integral_constant<int, -1>;
        using B = std::integral_constant<int, +1>;
        using AY = std::integral_constant<int, 1>;
        using AXc = std::integral_constant<int, 0>;
        if (dir < 0 && axis == 1) go(F{}, AY{});
        else if (dir < 0) go(F{}, AXc{});
        else if (axis == 1) go(B{}, AY{});
        else go(B{}, AXc{});
    }
    static void xgreen(const Plan& p, T* mesh, double cg, int nbox = 1) {
        C* d = reinterpret_cast<C*>(mesh);
        dim3 grid((H + TK - 1) / TK, N * nbox);
        Timed t(p, ST_FFT_X_GREEN);
        k_fft_x_green<T, N, TK, RV><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            d, (long long)N * H, H, (long long)N * N * H, H, static_cast<const C*>(p.tw),
            static_cast<const T*>(p.g1d), cg, p.green_kind, d);
    }
    // One box through the transposed spectrum `xt` ([ky][kx][kz], N^2 H
    // complex): x forward + Green + x inverse from `mesh` into `xt`, then the
    // inverse y pass from `xt` back into `mesh` ([x][y][kz]).
    static void xgreen_yinv_transposed(const Plan& p, T* mesh, T* xt, double cg) {
        C* d = reinterpret_cast<C*>(mesh);
        C* o = reinterpret_cast<C*>(xt);
        const C* tw = static_cast<const C*>(p.tw);
        const dim3 grid((H + TK - 1) / TK, N);
        {
            Timed t(p, ST_FFT_X_GREEN);
            k_fft_x_green<T, N, TK, RV, true><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
                d, (long long)N * H, H, (long long)N * N * H, H, tw, static_cast<const T*>(p.g1d), cg, p.green_kind,
                o);
        }
        Timed t(p, ST_FFT_Y_INV);
        k_fft_strided<T, N, +1, TK, RV, 2><<<grid, strided_threads<N, TK, RV>(), smem_s(), p.stream>>>(
            o, (long long)N * H, H, (long long)N * N * H, H, tw, d);
    }
};

#define PMB_FFT_DISPATCH(NG, ...)                                    \
    switch (NG) {                                                    \
        case 8: { constexpr int N_ = 8; __VA_ARGS__; } break;        \
        case 16: { constexpr int N_ = 16; __VA_ARGS__; } break;      \
        case 32: { constexpr int N_ = 32; __VA_ARGS__; } break;      \
        case 24: { constexpr int N_ = 24; __VA_ARGS__; } break;      \
        case 40: { constexpr int N_ = 40; __VA_ARGS__; } break;      \
        case 48: { constexpr int N_ = 48; __VA_ARGS__; } break;      \
        case 64: { constexpr int N_ = 64; __VA_ARGS__; } break;      \
        case 80: { constexpr int N_ = 80; __VA_ARGS__; } break;      \
        case 96: { constexpr int N_ = 96; __VA_ARGS__; } break;      \
        case 120: { constexpr int N_ = 120; __VA_ARGS__; } break;    \
        case 128: { constexpr int N_ = 128; __VA_ARGS__; } break;    \
        case 160: { constexpr int N_ = 160; __VA_ARGS__; } break;    \
        case 192: { constexpr int N_ = 192; __VA_ARGS__; } break;    \
        case 240: { constexpr int N_ = 240; __VA_ARGS__; } break;    \
        case 256: { constexpr int N_ = 256; __VA_ARGS__; } break;    \
        case 320: { constexpr int N_ = 320; __VA_ARGS__; } break;    \
        case 384: { constexpr int N_ = 384; __VA_ARGS__; } break;    \
        case 480: { constexpr int N_ = 480; __VA_ARGS__; } break;    \
        case 512: { constexpr int N_ = 512; __VA_ARGS__; } break;    \
        case 640: { constexpr int N_ = 640; __VA_ARGS__; } break;    \
        case 768: { constexpr int N_ = 768; __VA_ARGS__; } break;    \
        case 960: { constexpr int N_ = 960; __VA_ARGS__; } break;    \
        case 1024: { constexpr int N_ = 1024; __VA_ARGS__; } break;  \
        default: return fail(PM_ERR_SIZE, "mesh size not supported"); \
    }

// Powers of two 8..1024 and the mixed-radix sizes 2^a 3^b 5^c (multiples of
// 8, so that the FP32 deposit's 8^3 or 16^3 tiles divide the mesh).
bool fft_size_supported(int ng) {
    if (ng >= 8 && ng <= 1024 && (ng & (ng - 1)) == 0) return true;
    switch (ng) {
        case 24: case 40: case 48: case 80: case 96: case 120: case 160: case 192: case 240: case 320: case 384:
        case 480: case 640: case 768: case 960: return true;
        default: return false;
    }
}

// Launcher of a mesh size: the two-pass power-of-two kernels, or the
// generic mixed-radix ones for the 2^a 3^b 5^c sizes.
template <typename T, int N, int TK = 0, int RV = 0>
using LaunchFor = typename std::conditional<
    (N & (N - 1)) == 0, Launch<T, N, TK == 0 ? tk_cols<T, N>() : TK, RV>, LaunchG<T, N, TK == 0 ? gtk<T, N>() : TK>>::type;

// Column-tile widths the autotuner may pick for small FP32 meshes (ng <= 128);
// Plan::tk == 0 keeps the default width.
bool tk_variant_supported(int ng, int precision, int tk) {
    return tk == 0 || (precision == PM_FP32 && ng <= 128 && (tk == 8 || tk == 16 || tk == 32));
}

// The alternative radix split (RadixV<ng, 1>) exists for FP32 power-of-two
// meshes 16..128.
bool radix_variant_supported(int ng, int precision, int rv) {
    return rv == 0 || (rv == 1 && precision == PM_FP32 && ng >= 16 && ng <= 128 && (ng & (ng - 1)) == 0);
}

// First radix of the strided passes' two-pass split (0 for the mixed-radix
// mixed-radix schedules).
int strided_radix1(int ng, int rv) {
    switch (ng) {
        case 8: return Radix<8>::R1;
        case 16: return rv ? RadixV<16, 1>::R1 : Radix<16>::R1;
        case 32: return rv ? RadixV<32, 1>::R1 : Radix<32>::R1;
        case 64: return rv ? RadixV<64, 1>::R1 : Radix<64>::R1;
        case 128: return rv ? RadixV<128, 1>::R1 : Radix<128>::R1;
        case 256: return Radix<256>::R1;
        case 512: return Radix<512>::R1;
        case 1024: return Radix<1024>::R1;
        default: return 0;
    }
}

// Runs BODY with the launcher L_ of the plan's mesh size, tile width and
// radix split.
#define PMB_LAUNCH_TK(P, T_, RV_, ...)                                                                 \
    if ((P).tk == 8) { using L_ = LaunchFor<T_, N_, 8, RV_>; __VA_ARGS__; break; }                     \
    if ((P).tk == 16) { using L_ = LaunchFor<T_, N_, 16, RV_>; __VA_ARGS__; break; }                   \
    if ((P).tk == 32) { using L_ = LaunchFor<T_, N_, 32, RV_>; __VA_ARGS__; break; }                   \
    { using L_ = LaunchFor<T_, N_, 0, RV_>; __VA_ARGS__; break; }

#define PMB_LAUNCH(P, T_, ...)                                                                         \
    PMB_FFT_DISPATCH((P).ng, {                                                                         \
        if constexpr (sizeof(T_) == 4 && N_ <= 128) {                                                  \
            if constexpr (N_ >= 16 && (N_ & (N_ - 1)) == 0) {                                          \
                if ((P).rv == 1) { PMB_LAUNCH_TK(P, T_, 1, __VA_ARGS__) }                              \
            }                                                                                          \
            PMB_LAUNCH_TK(P, T_, 0, __VA_ARGS__)                                                       \
        }                                                                                              \
        using L_ = LaunchFor<T_, N_>;                                                                  \
        __VA_ARGS__;                                                                                   \
    })

int fft_prepare(const Plan& p) {
    int rc = PM_OK;
    if (p.precision == PM_FP64) {
        PMB_FFT_DISPATCH(p.ng, rc = LaunchFor<double, N_>::prepare());
    } else {
        PMB_FFT_DISPATCH(p.ng, {
            rc = LaunchFor<float, N_>::prepare();
            if constexpr (N_ <= 128) {
                if (rc == PM_OK) rc = LaunchFor<float, N_, 8>::prepare();
                if (rc == PM_OK) rc = LaunchFor<float, N_, 16>::prepare();
                if (rc == PM_OK) rc = LaunchFor<float, N_, 32>::prepare();
                if constexpr (N_ >= 16 && (N_ & (N_ - 1)) == 0) {
                    if (rc == PM_OK) rc = LaunchFor<float, N_, 0, 1>::prepare();
                    if (rc == PM_OK) rc = LaunchFor<float, N_, 8, 1>::prepare();
                    if (rc == PM_OK) rc = LaunchFor<float, N_, 16, 1>::prepare();
                    if (rc == PM_OK) rc = LaunchFor<float, N_, 32, 1>::prepare();
                }
            }
        });
    }
    return rc;
}

template <typename T> int fft_r2c(const Plan& p, T* mesh, int nbox) {
    PMB_LAUNCH(p, T, {
        L_::z(p, mesh, true, nbox);
        L_::strided(p, mesh, 1, -1, nbox);
        L_::strided(p, mesh, 0, -1, nbox);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template <typename T> int fft_c2r(const Plan& p, T* mesh, int nbox) {
    PMB_LAUNCH(p, T, {
        L_::strided(p, mesh, 0, +1, nbox);
        L_::strided(p, mesh, 1, +1, nbox);
        L_::z(p, mesh, false, nbox);
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
    Timed t(p, ST_GREEN);
    k_green<T><<<grid_for(p, (long long)p.ng * p.ng, 1), 256, 0, p.stream>>>(
        reinterpret_cast<C*>(mesh), p.ng, static_cast<const C*>(p.tw), static_cast<const T*>(p.g1d),
        green_scale(p, c_poisson), p.green_kind);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// The y forward, x + Green and y inverse passes of a solve (launcher L_):
// through the plan's transposed spectrum when it has one (a single box of a
// power-of-two mesh >= 512), else in place.
#define PMB_XY_PASSES(P, T_, MESH, CG, NBOX)                                   \
    L_::strided(P, MESH, 1, -1, NBOX);                                         \
    if (L_::kTransposedX && (NBOX) == 1 && (P).xspec) {                        \
        L_::xgreen_yinv_transposed(P, MESH, static_cast<T_*>((P).xspec), CG);  \
    } else {                                                                   \
        L_::xgreen(P, MESH, CG, NBOX);                                         \
        L_::strided(P, MESH, 1, +1, NBOX);                                     \
    }

template <typename T> int poisson_fused(const Plan& p, T* mesh, double c_poisson, int nbox) {
    const double cg = green_scale(p, c_poisson);
    PMB_LAUNCH(p, T, {
        L_::z(p, mesh, true, nbox);
        PMB_XY_PASSES(p, T, mesh, cg, nbox);
        L_::z(p, mesh, false, nbox);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int poisson_after_z_f32(const Plan& p, float* mesh, double c_poisson, int nbox) {
    const double cg = green_scale(p, c_poisson);
    PMB_LAUNCH(p, float, {
        PMB_XY_PASSES(p, float, mesh, cg, nbox);
        L_::z(p, mesh, false, nbox);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// ------------------------------------------------ x-slab decomposition
// The FFT passes of one slab (power-of-two FP32 meshes): the y forward pass
// over the slab's nx own planes (after the deposit's z R2C), the x forward +
// Green + x inverse over the nyl ky planes the slab holds after the global
// transpose, and the y inverse + z C2R over its own planes again.
#define PMB_SLAB_LAUNCH(P, ...)                                                    \
    PMB_FFT_DISPATCH((P).ng, {                                                     \
        if constexpr ((N_ & (N_ - 1)) == 0) {                                      \
            using L_ = Launch<float, N_>;                                          \
            __VA_ARGS__;                                                           \
        } else {                                                                   \
            return fail(PM_ERR_SIZE, "the slab path needs a power-of-two mesh");   \
        }                                                                          \
    })

int slab_fft_forward_y_f32(const Plan& p, const float* own, float* send, int nx) {
    PMB_SLAB_LAUNCH(p, L_::y_to_rows(p, own, send, nx));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int slab_fft_xgreen_f32(const Plan& p, const float* recv, float* send, double c_poisson, int nx, int ky0) {
    const double cg = green_scale(p, c_poisson);
    int nxl = 0;
    while ((1 << nxl) < nx) ++nxl;
    const int H = p.ng / 2 + 1;
    // rank kx / nx's block [kyl][x][kz]: (nx^2 H * (ng / nx) <= ng^2 H < 2^31)
    const LineMap m{(long long)nx * H, nx * nx * H, H, nxl, nx - 1};
    PMB_SLAB_LAUNCH(p, L_::xgreen_map(p, recv, send, cg, m, nx, H, ky0, 0));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int slab_fft_forward_peers_f32(const Plan& p, const float* own, const PeerMap& po, int nx) {
    PMB_SLAB_LAUNCH(p, L_::y_to_peers(p, own, po, nx));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int slab_fft_xgreen_peers_f32(const Plan& p, const float* recv, const PeerMap& po, double c_poisson, int nx,
                              int ky0) {
    const double cg = green_scale(p, c_poisson);
    int nxl = 0;
    while ((1 << nxl) < nx) ++nxl;
    const int H = p.ng / 2 + 1;
    const LineMap m{(long long)nx * H, nx * nx * H, H, nxl, nx - 1};
    PMB_SLAB_LAUNCH(p, L_::xgreen_peers(p, recv, cg, m, po, nx, H, ky0, 0));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int slab_fft_backward_f32(const Plan& p, const float* recv, float* own, int nx) {
    PMB_SLAB_LAUNCH(p, {
        L_::y_from_rows(p, recv, own, nx);
        L_::z_rows(p, own, false, (long long)nx * N_);
    });
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// ---------------------------------------------- pencil decomposition
// dst block [a][b][c] (strides da, db, 1) <- src block (strides sa, sb, 1),
// complex elements, one warp per (a, b) row with eight loads in flight per
// lane.  bg: subtracted from both halves of every element but a row's last
// (the density contrast's -1 background of the real rows; their last
// element is the z padding).
__global__ void k_copy3(const float2* __restrict__ src, long long sa, long long sb, float2* __restrict__ dst,
                        long long da, long long db, int B, long long rows, int Cn, float bg) {
    const int lane = threadIdx.x & 31;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const long long a = r / B, b = r - a * B;
        const float2* s = src + a * sa + b * sb;
        float2* d = dst + a * da + b * db;
        for (int e0 = lane; e0 < Cn; e0 += 32 * 8) {
            float2 v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (e0 + 32 * u < Cn) v[u] = __ldcs(s + e0 + 32 * u);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int c = e0 + 32 * u;
                if (c < Cn) d[c] = c < Cn - 1 ? make_float2(v[u].x - bg, v[u].y - bg) : v[u];
            }
        }
    }
}

int pencil_copy3(const Plan& p, const float2* src, long long sa, long long sb, float2* dst, long long da,
                 long long db, int A, int B, int C, float bg) {
    const long long rows = (long long)A * B;
    if (rows * C == 0) return PM_OK;
    k_copy3<<<grid_for(p, rows * 32, 256, 8), 256, 0, p.stream>>>(src, sa, sb, dst, da, db, B, rows, C, bg);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_lines_f32(const Plan& p, const float* in, float* out, LineMap mi, LineMap mo, int planes, int ncols,
                     int dir, int stage) {
    if (planes <= 0 || ncols <= 0) return PM_OK;
    PMB_SLAB_LAUNCH(p, L_::lines_map(p, in, out, mi, mo, planes, ncols, dir, stage));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_xgreen_f32(const Plan& p, const float* in, float* out, LineMap m, int planes, int ncols, double c_poisson,
                      int ky0, int kz0) {
    if (planes <= 0 || ncols <= 0) return PM_OK;
    const double cg = green_scale(p, c_poisson);
    PMB_SLAB_LAUNCH(p, L_::xgreen_map(p, in, out, cg, m, planes, ncols, ky0, kz0));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_lines_peers_f32(const Plan& p, const float* in, LineMap mi, const PeerMap& po, int planes, int ncols,
                           int dir, int stage) {
    if (planes <= 0 || ncols <= 0) return PM_OK;
    PMB_SLAB_LAUNCH(p, L_::lines_peers(p, in, mi, po, planes, ncols, dir, stage));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_xgreen_peers_f32(const Plan& p, const float* in, LineMap m, const PeerMap& po, int planes, int ncols,
                            double c_poisson, int ky0, int kz0) {
    if (planes <= 0 || ncols <= 0) return PM_OK;
    const double cg = green_scale(p, c_poisson);
    PMB_SLAB_LAUNCH(p, L_::xgreen_peers(p, in, cg, m, po, planes, ncols, ky0, kz0));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_z_f32(const Plan& p, float* rows, long long nrows, bool forward) {
    PMB_SLAB_LAUNCH(p, L_::z_rows(p, rows, forward, nrows));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

template int fft_r2c<float>(const Plan&, float*, int);
template int fft_r2c<double>(const Plan&, double*, int);
template int fft_c2r<float>(const Plan&, float*, int);
template int fft_c2r<double>(const Plan&, double*, int);
template int green_apply<float>(const Plan&, float*, double);
template int green_apply<double>(const Plan&, double*, double);
template int poisson_fused<float>(const Plan&, float*, double, int);
template int poisson_fused<double>(const Plan&, double*, double, int);

}  // namespace pmb
