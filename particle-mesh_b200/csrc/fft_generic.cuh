// Mixed-radix (3 x 2^k) FFT passes for the mesh sizes 48 and 96 of the
// batched-ensemble configuration.  A plain multi-pass Stockham schedule
// (the same autosort recurrence as fft_engine.cuh) over ping-pong shared
// buffers, with the radix list fixed per length:
//   24 = 3 x 8,  48 = 3 x 4 x 4,  96 = 3 x 4 x 8.
// The radix-3 butterfly is the one of FFTE (src/fft/ffte1/kernel.f:33-52, FFT3A):
// X0 = a + (b + c), X1,2 = a - (b + c)/2 -/+ sign i sqrt(3)/2 (b - c).
#pragma once

#include "fft_engine.cuh"

namespace pmb {

// In-register DFT of R in natural output order (R = 3 or a power of two).
template <int R, int DIR, typename C>
__device__ __forceinline__ void dft_nat(C* v) {
    using T = decltype(C::x);
    if constexpr (R == 3) {
        const C s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const C m = cmake<C>(v[0].x - (T)0.5 * s.x, v[0].y - (T)0.5 * s.y);
        constexpr T h = (T)0.86602540378443864676;  // sqrt(3)/2
        const C t = cmake<C>(-(T)DIR * h * d.y, (T)DIR * h * d.x);
        v[0] = cadd(v[0], s);
        v[1] = cadd(m, t);
        v[2] = csub(m, t);
    } else {
        dft<R, DIR>(v);
        C t[R];
#pragma unroll
        for (int k = 0; k < R; ++k) t[k] = v[brev<R>(k)];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = t[k];
    }
}

template <int L> struct GRadix;
template <> struct GRadix<24> {
    static constexpr int P = 2, NT = 8;
    static __host__ __device__ constexpr int R(int p) { return p == 0 ? 3 : 8; }
};
template <> struct GRadix<48> {
    static constexpr int P = 3, NT = 16;
    static __host__ __device__ constexpr int R(int p) { return p == 0 ? 3 : 4; }
};
template <> struct GRadix<96> {
    static constexpr int P = 3, NT = 32;
    static __host__ __device__ constexpr int R(int p) { return p == 0 ? 3 : (p == 1 ? 4 : 8); }
};

// One Stockham pass of radix R after Ns: in -> out, butterflies j = tj,
// tj + NT, ...; element e of a buffer lives at ix(e).  The twiddle
// W_L^e is tw[tws * e] (tws = N / L for a table of length N).
template <int L, int R, int DIR, typename C, typename IX>
__device__ __forceinline__ void gpass(const C* in, C* out, int Ns, int tj, int NT, const IX& ix,
                                      const C* __restrict__ tw, int tws) {
    for (int j = tj; j < L / R; j += NT) {
        C v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[ix(j + r * (L / R))];
        const int jm = j % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twiddle<DIR>(tw, tws * r * jm * (L / (Ns * R))));
        }
        dft_nat<R, DIR>(v);
        const int base = (j / Ns) * Ns * R + jm;
#pragma unroll
        for (int k = 0; k < R; ++k) out[ix(base + k * Ns)] = v[k];
    }
}

// All passes of length L; the result is in a (returned) or b.
template <int L, int DIR, typename C, typename IX>
__device__ __forceinline__ C* gfft(C* a, C* b, int tj, const IX& ix, const C* __restrict__ tw, int tws) {
    using G = GRadix<L>;
    C* in = a;
    C* out = b;
    int Ns = 1;
#pragma unroll
    for (int p = 0; p < G::P; ++p) {
        const int R = G::R(p);
        if (R == 3) gpass<L, 3, DIR>(in, out, Ns, tj, G::NT, ix, tw, tws);
        else if (R == 4) gpass<L, 4, DIR>(in, out, Ns, tj, G::NT, ix, tw, tws);
        else if (R == 8) gpass<L, 8, DIR>(in, out, Ns, tj, G::NT, ix, tw, tws);
        __syncthreads();
        Ns *= R;
        C* t = in;
        in = out;
        out = t;
    }
    return in;
}

}  // namespace pmb
