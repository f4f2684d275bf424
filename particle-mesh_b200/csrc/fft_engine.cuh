// Register-resident radix-R DFTs and the mixed-radix Stockham pass schedule
// used by every FFT kernel of the particle-mesh step.
//
// Stockham autosort (decimation in time), line length N = R1 * R2 * ...:
//   pass with radix R after Ns = product of earlier radices:
//     thread j in [0, N/R) reads v[r] = in[j + r N/R],
//     multiplies v[r] by W_N^{r (j mod Ns) N/(Ns R)},  W_N = exp(sign 2 pi i / N),
//     takes the radix-R DFT of v, and writes
//     out[(j / Ns) Ns R + (j mod Ns) + k Ns] = V[k].
// The output is in natural order after the last pass.  This is the same
// mixed-radix factorisation idea as the reference's FFTE kernels
// (src/fft/ffte1/fft235.f:20-121, twiddles fft235.f:205-219), reorganised so
// that one thread owns one radix-R butterfly held in registers.
#pragma once

#include <type_traits>

#include "pm_internal.cuh"

namespace pmb {

// cos / sin (2 pi k / 64), k = 0..31 (rounded to double).
__device__ __forceinline__ double cos64(int k) {
    constexpr double c[32] = {
        1.0, 0.9951847266721969, 0.9807852804032304, 0.9569403357322088, 0.9238795325112867,
        0.881921264348355, 0.8314696123025452, 0.773010453362737, 0.7071067811865476,
        0.6343932841636455, 0.5555702330196022, 0.47139673682599764, 0.3826834323650898,
        0.2902846772544624, 0.19509032201612828, 0.0980171403295606, 0.0, -0.0980171403295606,
        -0.19509032201612828, -0.2902846772544624, -0.3826834323650898, -0.47139673682599764,
        -0.5555702330196022, -0.6343932841636455, -0.7071067811865476, -0.773010453362737,
        -0.8314696123025452, -0.881921264348355, -0.9238795325112867, -0.9569403357322088,
        -0.9807852804032304, -0.9951847266721969};
    return c[k];
}
__device__ __forceinline__ double sin64(int k) { return k <= 16 ? cos64(16 - k) : cos64(k - 16); }

// d * exp(DIR 2 pi i k / 64), k a compile-time constant after unrolling.
template <int DIR, typename C>
__device__ __forceinline__ C rot64(C d, int k) {
    using T = decltype(C::x);
    constexpr T h = (T)0.7071067811865476;
    if (k == 0) return d;
    if (k == 16) return DIR < 0 ? cmake<C>(d.y, -d.x) : cmake<C>(-d.y, d.x);
    if (k == 8)
        return DIR < 0 ? cmake<C>((d.x + d.y) * h, (d.y - d.x) * h) : cmake<C>((d.x - d.y) * h, (d.x + d.y) * h);
    if (k == 24)
        return DIR < 0 ? cmake<C>((d.y - d.x) * h, -(d.x + d.y) * h) : cmake<C>(-(d.x + d.y) * h, (d.x - d.y) * h);
    const T c = (T)cos64(k), s = (T)(DIR * sin64(k));
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    if constexpr (sizeof(T) == 4)  // d.x (c, s) + d.y (-s, c) on the f32x2 pipe
        return __ffma2_rn(make_float2(d.y, d.y), make_float2(-s, c), __fmul2_rn(make_float2(d.x, d.x), make_float2(c, s)));
#endif
    return cmake<C>(d.x * c - d.y * s, d.x * s + d.y * c);
}

// Bit reversal of k on log2(R) bits.
template <int R>
__host__ __device__ constexpr int brev(int k) {
    int r = 0;
    for (int m = R >> 1, b = 1; m >= 1; m >>= 1, b <<= 1)
        if (k & m) r |= b;
    return r;
}

// In-register radix-R DFT (R a power of two <= 32), decimation in frequency;
// on return V[k] = v[brev<R>(k)].
template <int R, int DIR, typename C>
__device__ __forceinline__ void dft(C* v) {
#pragma unroll
    for (int half = R / 2; half >= 1; half >>= 1) {
#pragma unroll
        for (int b = 0; b < R; b += 2 * half) {
#pragma unroll
            for (int i = 0; i < half; ++i) {
                const C a = v[b + i], c = v[b + i + half];
                v[b + i] = cadd(a, c);
                v[b + i + half] = rot64<DIR>(csub(a, c), i * (64 / (2 * half)));
            }
        }
    }
}

// Twiddle W_N^e from the table tw[e] = exp(-2 pi i e / N) (inverse: conj).
template <int DIR, typename C>
__device__ __forceinline__ C twiddle(const C* __restrict__ tw, int e) {
    const C w = __ldg(tw + e);
    return DIR < 0 ? w : cconj(w);
}

// Pass-2 twiddles W_N^(S r j) of one thread (fixed j, r < 32; S = 2 for the
// half-length line of the z passes) from 10 table loads instead of 31:
// W^(S m j), m < 8, held in registers and W^(8 S q j) loaded per q,
// multiplied for r = 8 q + m (one extra complex product, ~1 ulp).
template <int DIR, typename C, int S = 1> struct TwSplit8 {
    const C* __restrict__ tw;
    int j;
    C wm[8];
    __device__ __forceinline__ TwSplit8(const C* __restrict__ tw_, int j_) : tw(tw_), j(j_) {
        wm[0] = cmake<C>(1, 0);
#pragma unroll
        for (int m = 1; m < 8; ++m) wm[m] = twiddle<DIR>(tw, S * m * j);
    }
    __device__ __forceinline__ C operator()(int r, int) const {
        const int q = r >> 3, m = r & 7;
        if (q == 0) return wm[m];
        const C b = twiddle<DIR>(tw, 8 * S * q * j);
        return m == 0 ? b : cmul(b, wm[m]);
    }
};

// The pass-2 twiddle functor of thread j: split (TwSplit8, needs R2 >= 16 so
// that every index stays below L = R1 R2) or one table load per twiddle.
template <int DIR, bool SPLIT, int S = 1, typename C>
__device__ __forceinline__ auto pass2_twiddles(const C* __restrict__ tw, int j) {
    if constexpr (SPLIT)
        return TwSplit8<DIR, C, S>(tw, j);
    else
        return [tw](int e) { return twiddle<DIR>(tw, S * e); };
}

// Two-pass radix choice for a line of length L = R1 * R2, R1 <= R2.
template <int L> struct Radix;
template <> struct Radix<4> { static constexpr int R1 = 2, R2 = 2; };
template <> struct Radix<8> { static constexpr int R1 = 2, R2 = 4; };
template <> struct Radix<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Radix<32> { static constexpr int R1 = 4, R2 = 8; };
template <> struct Radix<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Radix<128> { static constexpr int R1 = 8, R2 = 16; };
template <> struct Radix<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Radix<512> { static constexpr int R1 = 16, R2 = 32; };
template <> struct Radix<1024> { static constexpr int R1 = 32, R2 = 32; };

// Threads per line: one radix-R2 butterfly each in pass 2; pass 1 has
// R2 / R1 radix-R1 butterflies per thread.
template <int L> constexpr int threads_per_line() { return L / Radix<L>::R2; }

// Split variants of a strided line for the autotuner: RV = 0 is Radix<L>,
// RV = 1 a smaller first radix and a larger second one (more work per
// thread, fewer threads per line), still with R2 % R1 == 0.
template <int L, int RV> struct RadixV : Radix<L> {};
template <> struct RadixV<16, 1> { static constexpr int R1 = 2, R2 = 8; };
template <> struct RadixV<32, 1> { static constexpr int R1 = 2, R2 = 16; };
template <> struct RadixV<64, 1> { static constexpr int R1 = 4, R2 = 16; };
template <> struct RadixV<128, 1> { static constexpr int R1 = 4, R2 = 32; };
template <int L, int RV> constexpr int threads_per_line_v() { return L / RadixV<L, RV>::R2; }

// Stockham pass 1 (Ns = 1, radix R1) of a line of L = R1 R2: thread tj owns
// the butterflies j = tj + it R1 (it < R2/R1).  ld(j, r) returns element
// j + r R2; st(j, k, v) stores output k of butterfly j, element j R1 + k.
// The structured indices let each kernel form its (padded) addresses as a
// per-j base plus compile-time offsets.  With SYNC the block synchronises
// between all loads and all stores (in-place passes).
template <int R1, int R2, int DIR, bool SYNC, typename C, typename LD, typename ST>
__device__ __forceinline__ void stockham_pass1(int tj, const LD& ld, const ST& st) {
    constexpr int IT = R2 / R1;
    C v[IT][R1];
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = tj + it * R1;
#pragma unroll
        for (int r = 0; r < R1; ++r) v[it][r] = ld(j, r);
        dft<R1, DIR>(v[it]);
    }
    if (SYNC) __syncthreads();
#pragma unroll
    for (int it = 0; it < IT; ++it) {
        const int j = tj + it * R1;
#pragma unroll
        for (int k = 0; k < R1; ++k) st(j, k, v[it][brev<R1>(k)]);
    }
}

// Stockham pass 2 (Ns = R1, radix R2): thread j < R1 reads ld(j, r) =
// element j + r R1, multiplies by W_L^{r j} (twf(r j)) and stores output k
// with st(j, k, v) to element j + k R1.
template <int R1, int R2, int DIR, bool SYNC, typename C, typename LD, typename ST, typename TW>
__device__ __forceinline__ void stockham_pass2(int j, const LD& ld, const ST& st, const TW& twf) {
    C v[R2];
#pragma unroll
    for (int r = 0; r < R2; ++r) v[r] = ld(j, r);
#pragma unroll
    for (int r = 1; r < R2; ++r) {
        if constexpr (std::is_invocable_v<const TW&, int, int>)
            v[r] = cmul(v[r], twf(r, j));
        else
            v[r] = cmul(v[r], twf(r * j));
    }
    dft<R2, DIR>(v);
    if (SYNC) __syncthreads();
#pragma unroll
    for (int k = 0; k < R2; ++k) st(j, k, v[brev<R2>(k)]);
}

// Padded shared-memory index of the z passes: one pad entry after every R1
// entries, so the pass-1 writes j*R1 + k of consecutive j hit distinct banks.
template <int R1> __device__ __forceinline__ int zpad(int i) { return i + i / R1; }
// The same positions as base + compile-time offset for the two-pass schedule
// (L = R1 R2, R2 % R1 == 0): pass-1 input j + r R2, pass-1 output j R1 + k,
// pass-2 input / output j + r R1 (j < R1).
template <int R1, int R2> struct ZIdx {  // z passes, unit stride, pad 1 per R1
    static __device__ __forceinline__ int in1(int j, int r) { return j + j / R1 + r * (R2 + R2 / R1); }
    static __device__ __forceinline__ int out1(int j, int k) { return j * (R1 + 1) + k; }
    static __device__ __forceinline__ int p2(int j, int r) { return j + r * (R1 + 1); }
};
// Post-processing of the z R2C from the registers of pass 2.  Thread tj of
// a row (R1 threads per row, lanes tj of one aligned group of R1 in a warp)
// holds Z[tj + R1 k] in X[k]; output m = tj + R1 k needs Z[M - m], which is
// X[R2 - 1 - k] of lane R1 - tj (or, for tj = 0, its own X[(R2 - k) mod R2]),
// fetched with one shuffle per element.  Writes the M + 1 spectrum entries
//   X[m] = E + W_N^m O,  E = (Z[m] + conj Z[M-m]) / 2,  O = -i (Z[m] - conj Z[M-m]) / 2
// (Z[M] taken as Z[0]); for fixed k the R1 lanes write consecutive entries.
template <int R1, int R2, typename C>
__device__ __forceinline__ void r2c_post(const C (&X)[R2], int tj, bool active, C* __restrict__ crow,
                                         const C* __restrict__ tw) {
    using T = decltype(C::x);
    constexpr int M = R1 * R2;
    const int partner = (R1 - tj) & (R1 - 1);
#pragma unroll
    for (int k = 0; k < R2; ++k) {
        const C q = X[R2 - 1 - k];
        C p;
        p.x = __shfl_sync(0xffffffffu, q.x, partner, R1);
        p.y = __shfl_sync(0xffffffffu, q.y, partner, R1);
        const C zc = cconj(tj == 0 ? X[(R2 - k) & (R2 - 1)] : p);
        const C zk = X[k];
        const C e = cscale(cadd(zk, zc), (T)0.5);
        const C d = csub(zk, zc);
        const C o = cmake<C>((T)0.5 * d.y, (T)-0.5 * d.x);  // -i d / 2
        const int m = tj + R1 * k;
        if (active) crow[m] = cadd(e, cmul(twiddle<-1>(tw, m), o));
    }
    if (active && tj == 0) {  // m = M: Z[M] = Z[0], W_N^M = -1
        const C zk = X[0], zc = cconj(X[0]);
        const C e = cscale(cadd(zk, zc), (T)0.5);
        const C d = csub(zk, zc);
        crow[M] = cmake<C>(e.x - (T)0.5 * d.y, e.y + (T)0.5 * d.x);
    }
}

// Complex entries per padded z row (M + 1 values of the half spectrum).
template <int N> constexpr int z_row_stride() { return (N / 2 + 1) + (N / 2 + 1) / Radix<N / 2>::R1 + 1; }

}  // namespace pmb
