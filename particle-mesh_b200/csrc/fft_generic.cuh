// Mixed-radix FFT passes for mesh sizes 2^a 3^b 5^c that are not powers of
// two (24 to 960, multiples of 8).  A plain multi-pass Stockham schedule (the
// same autosort recurrence as fft_engine.cuh) over ping-pong shared buffers.
// The line length is factored into radices 8, 5, 4, 3, 2 -- the radix set of
// the reference's FFTE (src/fft/ffte1/factor.f:19-43, kernel.f FFT2..FFT8) --
// with the 5s and 3s first, then as many 8s as fit, then one 4 or 2.
// The radix-3 and radix-5 butterflies are the published DFT identities that
// FFTE's FFT3A / FFT5A (src/fft/ffte1/kernel.f) also evaluate:
//   radix 3: X0 = a + (b + c), X1,2 = a - (b + c)/2 -/+ sign i sqrt(3)/2 (b - c);
//   radix 5: with t1 = x1 + x4, t2 = x2 + x3, t3 = x1 - x4, t4 = x2 - x3,
//            X0 = x0 + t1 + t2,
//            X1,4 = x0 + c1 t1 + c2 t2 +/- sign i (s1 t3 + s2 t4),
//            X2,3 = x0 + c2 t1 + c1 t2 +/- sign i (s2 t3 - s1 t4),
//            c1 = cos 2pi/5, c2 = cos 4pi/5, s1 = sin 2pi/5, s2 = sin 4pi/5.
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
    } else if constexpr (R == 5) {
        constexpr T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
        constexpr T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
        const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const C a1 = cmake<C>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
        const C a2 = cmake<C>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
        const C b1 = cmake<C>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        const C b2 = cmake<C>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        const C ib1 = cmake<C>(-(T)DIR * b1.y, (T)DIR * b1.x), ib2 = cmake<C>(-(T)DIR * b2.y, (T)DIR * b2.x);
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, ib1);
        v[4] = csub(a1, ib1);
        v[2] = cadd(a2, ib2);
        v[3] = csub(a2, ib2);
    } else {
        dft<R, DIR>(v);
        C t[R];
#pragma unroll
        for (int k = 0; k < R; ++k) t[k] = v[brev<R>(k)];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = t[k];
    }
}

// Radix schedule of a line of L = 2^a 3^b 5^c: all 5s, all 3s, then the
// power of two as 8s with one 4 for a remainder of 4, or two 4s for a
// remainder of 2 (a lone 2 only for a = 1).  NT threads per line: a power of
// two near a third of the line, at most 32.
namespace gr {
constexpr int pow_of(int L, int f) { return L % f == 0 ? 1 + pow_of(L / f, f) : 0; }
constexpr int n8(int a) { return a % 3 == 1 && a >= 4 ? (a - 4) / 3 : a / 3; }
constexpr int n4(int a) { return a % 3 == 2 ? 1 : (a % 3 == 1 && a >= 4 ? 2 : 0); }
constexpr int n2(int a) { return a == 1 ? 1 : 0; }
constexpr int radix_at(int L, int p) {
    const int a = pow_of(L, 2), f5 = pow_of(L, 5), f3 = pow_of(L, 3);
    if (p < f5) return 5;
    if (p < f5 + f3) return 3;
    const int q = p - f5 - f3;
    if (q < n8(a)) return 8;
    if (q < n8(a) + n4(a)) return 4;
    return 2;
}
constexpr int passes(int L) {
    const int a = pow_of(L, 2);
    return pow_of(L, 5) + pow_of(L, 3) + n8(a) + n4(a) + n2(a);
}
constexpr int threads(int L) {
    int t = 1;
    while (t * 2 <= L / 3 && t < 32) t *= 2;
    return t;
}
}  // namespace gr

template <int L> struct GRadix {
    static constexpr int P = gr::passes(L), NT = gr::threads(L);
    static __host__ __device__ constexpr int R(int p) { return gr::radix_at(L, p); }
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
        else if (R == 5) gpass<L, 5, DIR>(in, out, Ns, tj, G::NT, ix, tw, tws);
        else if (R == 2) gpass<L, 2, DIR>(in, out, Ns, tj, G::NT, ix, tw, tws);
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
