// Particle <-> mesh kernels of the particle-mesh step: CIC deposit, mesh
// gradient, CIC interpolation + kick, drift, and the FP32 split-position
// forms of the same.
//
// Periodic single box: the reference's ghost planes (+1 for the deposit,
// src/utils/utils.cpp:38-68 and src/decomp/slab/reorder_slab.cpp:3-68;
// -1/+2 for the gradient, src/decomp/slab/reorder_slab_back.cpp:3-49 and
// transpose_slab_back.cpp:3-49) become index wraps; ng is a power of two so a
// wrap is a mask.
#include <type_traits>

#include "pm_internal.cuh"

namespace pmb {

namespace {

// A position outside [0, n) (or NaN / inf) is recorded in the plan's error
// word and wrapped (NaN and inf -> 0) so that every access stays in bounds.
__device__ __forceinline__ double sanitize(double v, double n, int* err) {
    if (v >= 0.0 && v < n) return v;
    atomicOr(err, ERRBIT_RANGE);
    if (!isfinite(v)) return 0.0;
    double m = v - n * floor(v / n);
    if (m >= n) m -= n;
    if (m < 0.0) m = 0.0;
    return m;
}

__device__ __forceinline__ double wrap_pos(double v, double n) {
    v = v - n * floor(v / n);
    return v >= n ? v - n : v;  // v/n rounding can land exactly on n
}

// Every cell of a padded mesh [n][n][n+2] to val, padding to 0.  The mesh
// is a flat array of n^2 (n+2) values (a multiple of 4 for n >= 8) written
// as aligned 16-byte vectors; the allocation is 256-byte aligned.
template <typename T>
__global__ void k_mesh_init(T* __restrict__ mesh, int n, T val) {
    constexpr int W = 16 / sizeof(T);  // values per 16-byte vector
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    V* mv = reinterpret_cast<V*>(mesh);
    const unsigned pz = (unsigned)n + 2u;
    const unsigned long long total = (unsigned long long)n * n * pz / W;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < total;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned z0 = (unsigned)((i * W) % pz);
        T v[W];
#pragma unroll
        for (int c = 0; c < W; ++c) {
            unsigned z = z0 + c;
            z = z >= pz ? z - pz : z;
            v[c] = z < (unsigned)n ? val : (T)0;
        }
        V out;
        memcpy(&out, v, sizeof(V));
        mv[i] = out;
    }
}

// Neighbour index c in [-n, 2n) wrapped into [0, n): a mask for power-of-
// two meshes, one conditional otherwise (the mixed-radix sizes).
template <bool POW2>
__device__ __forceinline__ int wrap_near(int c, int n) {
    if (POW2) return c & (n - 1);
    return c < 0 ? c + n : (c >= n ? c - n : c);
}

// ------------------------------------------------------------------- FP64

// CIC deposit, one thread per particle, 8 FP64 atomics into the periodic
// mesh.  Same weights and operation order as cic_deposit
// (include/utils/utils_inline.h:25-49); cell = floor(x) as static_cast<int>
// in deposit_particles (src/utils/utils.cpp:85-97) for x >= 0.
template <bool POW2>
__global__ void k_deposit_f64(const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, long long np, double mass,
                              double* __restrict__ mesh, int n, int* err) {
    const double dn = (double)n;
    const long long pz = n + 2;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        const double xp = sanitize(x[p], dn, err), yp = sanitize(y[p], dn, err), zp = sanitize(z[p], dn, err);
        const double fx = floor(xp), fy = floor(yp), fz = floor(zp);
        const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
        const int i1 = wrap_near<POW2>(i0 + 1, n), j1 = wrap_near<POW2>(j0 + 1, n), k1 = wrap_near<POW2>(k0 + 1, n);
        const double tx = xp - fx, ty = yp - fy, tz = zp - fz;
        const double sx0 = 1.0 - tx, sy0 = 1.0 - ty, sz0 = 1.0 - tz;
        const double sxy00 = sx0 * sy0, sxy10 = tx * sy0, sxy01 = sx0 * ty, sxy11 = tx * ty;
        const double m0 = mass * sz0, m1 = mass * tz;
        const long long r00 = ((long long)i0 * n + j0) * pz, r10 = ((long long)i1 * n + j0) * pz;
        const long long r01 = ((long long)i0 * n + j1) * pz, r11 = ((long long)i1 * n + j1) * pz;
        atomicAdd(mesh + r00 + k0, sxy00 * m0);
        atomicAdd(mesh + r10 + k0, sxy10 * m0);
        atomicAdd(mesh + r01 + k0, sxy01 * m0);
        atomicAdd(mesh + r11 + k0, sxy11 * m0);
        atomicAdd(mesh + r00 + k1, sxy00 * m1);
        atomicAdd(mesh + r10 + k1, sxy10 * m1);
        atomicAdd(mesh + r01 + k1, sxy01 * m1);
        atomicAdd(mesh + r11 + k1, sxy11 * m1);
    }
}

// f = -grad phi by centred differences.  One block iteration per mesh row
// (i, j), threads along k, so the ten neighbour rows are addressed once.
//   order 2: (phi[i-1] - phi[i+1]) / 2          (src/utils/utils.cpp:130-135)
//   order 4: (8 (phi[i-1] - phi[i+1]) - (phi[i-2] - phi[i+2])) / 12
template <int ORDER, bool POW2>
__global__ void k_gradient_f64(const double* __restrict__ phi, double* __restrict__ fx,
                               double* __restrict__ fy, double* __restrict__ fz, int n) {
    const long long pz = n + 2;
    for (long long row = blockIdx.x; row < (long long)n * n; row += gridDim.x) {
        const int i = (int)(row / n), j = (int)(row % n);
        auto R = [&](int a, int b) {
            return phi + ((long long)wrap_near<POW2>(a, n) * n + wrap_near<POW2>(b, n)) * pz;
        };
        const double *c0 = R(i, j), *xm1 = R(i - 1, j), *xp1 = R(i + 1, j), *ym1 = R(i, j - 1), *yp1 = R(i, j + 1);
        const double *xm2 = R(i - 2, j), *xp2 = R(i + 2, j), *ym2 = R(i, j - 2), *yp2 = R(i, j + 2);
        const long long o = row * n;
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            const int km1 = wrap_near<POW2>(k - 1, n), kp1 = wrap_near<POW2>(k + 1, n);
            if (ORDER == 4) {
                const int km2 = wrap_near<POW2>(k - 2, n), kp2 = wrap_near<POW2>(k + 2, n);
                fx[o + k] = (8.0 * (__ldg(xm1 + k) - __ldg(xp1 + k)) - (__ldg(xm2 + k) - __ldg(xp2 + k))) / 12.0;
                fy[o + k] = (8.0 * (__ldg(ym1 + k) - __ldg(yp1 + k)) - (__ldg(ym2 + k) - __ldg(yp2 + k))) / 12.0;
                fz[o + k] = (8.0 * (__ldg(c0 + km1) - __ldg(c0 + kp1)) - (__ldg(c0 + km2) - __ldg(c0 + kp2))) / 12.0;
            } else {
                fx[o + k] = (__ldg(xm1 + k) - __ldg(xp1 + k)) * 0.5;
                fy[o + k] = (__ldg(ym1 + k) - __ldg(yp1 + k)) * 0.5;
                fz[o + k] = (__ldg(c0 + km1) - __ldg(c0 + kp1)) * 0.5;
            }
        }
    }
}

// Trilinear gather with the operation order of trilerp1
// (include/utils/utils_inline.h:55-70).
__device__ __forceinline__ double trilerp(const double* __restrict__ f, long long b00, long long b10,
                                          long long b01, long long b11, int k0, int k1, double tx,
                                          double ty, double tz) {
    const double mx = 1.0 - tx, my = 1.0 - ty, mz = 1.0 - tz;
    const double f00 = __ldg(f + b00 + k0) * mx + __ldg(f + b10 + k0) * tx;
    const double f10 = __ldg(f + b01 + k0) * mx + __ldg(f + b11 + k0) * tx;
    const double fz0 = f00 * my + f10 * ty;
    const double g00 = __ldg(f + b00 + k1) * mx + __ldg(f + b10 + k1) * tx;
    const double g10 = __ldg(f + b01 + k1) * mx + __ldg(f + b11 + k1) * tx;
    const double fz1 = g00 * my + g10 * ty;
    return fz0 * mz + fz1 * tz;
}

// p += c_kick * W^T f (update_particles, src/utils/utils.cpp:141-170).
template <bool POW2>
__global__ void k_interp_kick_f64(const double* __restrict__ x, const double* __restrict__ y,
                                  const double* __restrict__ z, const double* __restrict__ fx,
                                  const double* __restrict__ fy, const double* __restrict__ fz,
                                  double* __restrict__ px, double* __restrict__ py,
                                  double* __restrict__ pzv, long long np, double c_kick, int n,
                                  int* err) {
    const double dn = (double)n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        const double xp = sanitize(x[p], dn, err), yp = sanitize(y[p], dn, err), zp = sanitize(z[p], dn, err);
        const double flx = floor(xp), fly = floor(yp), flz = floor(zp);
        const int i0 = (int)flx, j0 = (int)fly, k0 = (int)flz;
        const int i1 = wrap_near<POW2>(i0 + 1, n), j1 = wrap_near<POW2>(j0 + 1, n), k1 = wrap_near<POW2>(k0 + 1, n);
        const double tx = xp - flx, ty = yp - fly, tz = zp - flz;
        const long long b00 = ((long long)i0 * n + j0) * n, b10 = ((long long)i1 * n + j0) * n;
        const long long b01 = ((long long)i0 * n + j1) * n, b11 = ((long long)i1 * n + j1) * n;
        px[p] += trilerp(fx, b00, b10, b01, b11, k0, k1, tx, ty, tz) * c_kick;
        py[p] += trilerp(fy, b00, b10, b01, b11, k0, k1, tx, ty, tz) * c_kick;
        pzv[p] += trilerp(fz, b00, b10, b01, b11, k0, k1, tx, ty, tz) * c_kick;
    }
}

__global__ void k_drift_f64(double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                            const double* __restrict__ px, const double* __restrict__ py,
                            const double* __restrict__ pz, long long np, double dt, int n) {
    const double dn = (double)n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        x[p] = wrap_pos(x[p] + px[p] * dt, dn);
        y[p] = wrap_pos(y[p] + py[p] * dt, dn);
        z[p] = wrap_pos(z[p] + pz[p] * dt, dn);
    }
}

// ------------------------------------------------------ split positions

__device__ __forceinline__ void split1(double v, int n, int& cell, float& off) {
    const double f = floor(v);
    cell = wrap_cell((int)(long long)f, n);
    off = (float)(v - f);
    if (off >= 1.0f) {  // rounding to FP32 reached the next cell
        off = 0.0f;
        cell = wrap_cell(cell + 1, n);
    }
}

__device__ __forceinline__ uint32_t pack_cell(int i, int j, int k) {
    return ((uint32_t)i << 20) | ((uint32_t)j << 10) | (uint32_t)k;
}
__device__ __forceinline__ void unpack_cell(uint32_t c, int& i, int& j, int& k) {
    i = (int)(c >> 20);
    j = (int)((c >> 10) & 1023u);
    k = (int)(c & 1023u);
}

__global__ void k_split(const double* __restrict__ x, const double* __restrict__ y,
                        const double* __restrict__ z, long long np, uint32_t* __restrict__ cell,
                        float* __restrict__ ox, float* __restrict__ oy, float* __restrict__ oz, int n,
                        int* err) {
    const double dn = (double)n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        float a, b, c;
        split1(sanitize(x[p], dn, err), n, i, a);
        split1(sanitize(y[p], dn, err), n, j, b);
        split1(sanitize(z[p], dn, err), n, k, c);
        cell[p] = pack_cell(i, j, k);
        ox[p] = a;
        oy[p] = b;
        oz[p] = c;
    }
}

__global__ void k_join(const uint32_t* __restrict__ cell, const float* __restrict__ ox,
                       const float* __restrict__ oy, const float* __restrict__ oz, long long np,
                       double* __restrict__ x, double* __restrict__ y, double* __restrict__ z) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(cell[p], i, j, k);
        x[p] = (double)i + (double)ox[p];
        y[p] = (double)j + (double)oy[p];
        z[p] = (double)k + (double)oz[p];
    }
}

// ------------------------------------------------------------------- FP32

// Force at one particle with the gradient fused into the gather: the
// trilinear weights of cells (i+a, j+b, k+c), a,b,c in {0,1}, applied to the
// centred difference of phi at those cells (2- or 4-point).  The stencils
// of the three components share their cells: each of the 32 (2-point) or 56
// (4-point) distinct values is loaded once, from 12 or 20 mesh rows whose
// offsets fit in 32 bits (ng <= 1024).

// The potential values the 2- or 4-point centred differences need at the 8
// CIC corners (i+a, j+b, k+c), each loaded once: the core rows (i+a, j+b)
// over the whole z stencil, and the x and y stencil rows at columns k, k+1.
// XPLAIN: the x planes are not periodic -- phi is one slab of a decomposed
// mesh with its halo planes, and i already indexes the buffer's planes.
// YPLAIN likewise for y: phi is one pencil with its halo rows, `yrows` rows
// per x plane, and j indexes the buffer's rows.
template <int ORDER, bool POW2, bool XPLAIN = false, bool YPLAIN = false> struct Stencil {
    static constexpr int LO = ORDER == 4 ? -2 : -1, W = ORDER == 4 ? 6 : 4;  // offsets LO..LO+W-1
    static constexpr int C0 = -LO;                                            // slot of offset 0
    float Z[2][2][W], X[W][2][2], Y[2][W][2];

    __device__ __forceinline__ Stencil(const float* __restrict__ phi, int n, int i, int j, int k, int yrows = 0) {
        const unsigned pz = (unsigned)n + 2u, plane = (unsigned)(YPLAIN ? yrows : n) * pz;
        unsigned xo[W], yo[W], kc[W];
#pragma unroll
        for (int d = 0; d < W; ++d) {
            xo[d] = (unsigned)(XPLAIN ? i + LO + d : wrap_near<POW2>(i + LO + d, n)) * plane;
            yo[d] = (unsigned)(YPLAIN ? j + LO + d : wrap_near<POW2>(j + LO + d, n)) * pz;
            kc[d] = (unsigned)wrap_near<POW2>(k + LO + d, n);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < W; ++c) Z[a][b][c] = __ldg(phi + xo[C0 + a] + yo[C0 + b] + kc[c]);
#pragma unroll
        for (int d = 0; d < W; ++d)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (d == C0 || d == C0 + 1) {
                        X[d][b][c] = Z[d - C0][b][C0 + c];
                        Y[b][d][c] = Z[b][d - C0][C0 + c];
                    } else {
                        X[d][b][c] = __ldg(phi + xo[d] + yo[C0 + b] + kc[C0 + c]);
                        Y[b][d][c] = __ldg(phi + xo[C0 + b] + yo[d] + kc[C0 + c]);
                    }
                }
    }
    // centred difference (minus the gradient) at slot s of a stencil line v
    static __device__ __forceinline__ float D(const float* v, int s) {
        return ORDER == 4 ? (8.0f * (v[s - 1] - v[s + 1]) - (v[s - 2] - v[s + 2])) * (1.0f / 12.0f)
                          : (v[s - 1] - v[s + 1]) * 0.5f;
    }
    // the three components of -grad phi at corner (a, b, c)
    __device__ __forceinline__ void corner(int a, int b, int c, float& fx, float& fy, float& fz) const {
        float lx[W], ly[W];
#pragma unroll
        for (int d = 0; d < W; ++d) {
            lx[d] = X[d][b][c];
            ly[d] = Y[a][d][c];
        }
        fx = D(lx, C0 + a);
        fy = D(ly, C0 + b);
        fz = D(Z[a][b], C0 + c);
    }
};

// Cell indices of a caller-provided cell word reduced into [0, n) (a word
// from pm_split_positions already is), so every mesh access stays in bounds.
// Power-of-two meshes need nothing here: every index is masked where used.
template <bool POW2>
__device__ __forceinline__ void canon_cell(int& i, int& j, int& k, int n) {
    if (!POW2) {
        if (i >= n) i %= n;
        if (j >= n) j %= n;
        if (k >= n) k %= n;
    }
}

// The same 56 (or 32) values from a block's staged potential in shared
// memory: rows of (x, y) on a square of side RW, z at padded index
// zp(z) = z + z / 32 within a row of RL floats (lanes two cells apart in z
// then fall on distinct banks).
template <int ORDER, int RW, int RL> struct SmemStencil {
    static constexpr int LO = ORDER == 4 ? -2 : -1, W = ORDER == 4 ? 6 : 4, C0 = -LO;
    float Z[2][2][W], X[W][2][2], Y[2][W][2];
    static __device__ __forceinline__ float D(const float* v, int s) {
        return ORDER == 4 ? (8.0f * (v[s - 1] - v[s + 1]) - (v[s - 2] - v[s + 2])) * (1.0f / 12.0f)
                          : (v[s - 1] - v[s + 1]) * 0.5f;
    }
    __device__ __forceinline__ SmemStencil(const float* __restrict__ S, int lx, int ly, int lz) {
        int xo[W], yo[W], kc[W];
#pragma unroll
        for (int d = 0; d < W; ++d) {
            xo[d] = (lx + LO + d) * (RW * RL);
            yo[d] = (ly + LO + d) * RL;
            const int z = lz + LO + d;
            kc[d] = z + (z >> 5);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < W; ++c) Z[a][b][c] = S[xo[C0 + a] + yo[C0 + b] + kc[c]];
#pragma unroll
        for (int d = 0; d < W; ++d)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (d == C0 || d == C0 + 1) {
                        X[d][b][c] = Z[d - C0][b][C0 + c];
                        Y[b][d][c] = Z[b][d - C0][C0 + c];
                    } else {
                        X[d][b][c] = S[xo[d] + yo[C0 + b] + kc[C0 + c]];
                        Y[b][d][c] = S[xo[C0 + b] + yo[d] + kc[C0 + c]];
                    }
                }
    }
};

// -grad phi interpolated at in-cell offsets (tx, ty, tz) from a stencil's
// values (Stencil or SmemStencil).
template <class St>
__device__ __forceinline__ void force_from(const St& s, float tx, float ty, float tz, float& gx, float& gy,
                                           float& gz) {
    constexpr int W = St::W, C0 = St::C0;
    const float w0[2] = {1.0f - tx, tx}, w1[2] = {1.0f - ty, ty}, w2[2] = {1.0f - tz, tz};
    gx = gy = gz = 0.0f;
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            float lx[W], ly[W];
#pragma unroll
            for (int d = 0; d < W; ++d) {
                lx[d] = s.X[d][b][c];
                ly[d] = s.Y[b][d][c];
            }
            gx += w1[b] * w2[c] * (w0[0] * St::D(lx, C0) + w0[1] * St::D(lx, C0 + 1));
            // for y the roles are (a = b here, c): weights w0[a] w2[c]
            gy += w0[b] * w2[c] * (w1[0] * St::D(ly, C0) + w1[1] * St::D(ly, C0 + 1));
        }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
            gz += w0[a] * w1[b] * (w2[0] * St::D(s.Z[a][b], C0) + w2[1] * St::D(s.Z[a][b], C0 + 1));
}

template <int ORDER, bool POW2, bool XPLAIN = false>
__device__ __forceinline__ void force_at(const float* __restrict__ phi, int n, int i, int j, int k,
                                         float tx, float ty, float tz, float& gx, float& gy,
                                         float& gz) {
    const Stencil<ORDER, POW2, XPLAIN> s(phi, n, i, j, k);
    force_from(s, tx, ty, tz, gx, gy, gz);
}

template <int ORDER, bool POW2>
__global__ void __launch_bounds__(256, 4) k_interp_f32(const float* __restrict__ phi, const uint32_t* __restrict__ cell,
                             const float* __restrict__ ox, const float* __restrict__ oy,
                             const float* __restrict__ oz, long long np, float* __restrict__ fx,
                             float* __restrict__ fy, float* __restrict__ fz, int n) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(__ldg(cell + p), i, j, k);
        canon_cell<POW2>(i, j, k, n);
        float gx, gy, gz;
        force_at<ORDER, POW2>(phi, n, i, j, k, __ldg(ox + p), __ldg(oy + p), __ldg(oz + p), gx, gy, gz);
        fx[p] = gx;
        fy[p] = gy;
        fz[p] = gz;
    }
}

// v += c_kick * force; x += dt * v accumulated in FP64 and re-split.
// Batches: with pbeg != null, grid row blockIdx.y advances the particles
// [pbeg[b], pend[b]) of box b in the mesh phi + b * mesh_stride.
// (at most 64 registers: four 256-thread blocks per SM keep enough warps in
// flight for the ~60 outstanding gathers per particle)
// SLAB: phi is one x-slab [x0, x0 + nxl) of the mesh with two halo planes
// below and three above (buffer plane = x - x0 + 2); a particle outside the
// slab is recorded in *err and clamped into it.
template <int ORDER, bool POW2, bool SLAB = false>
__global__ void __launch_bounds__(256, 4) k_kick_drift_f32(const float* __restrict__ phi, uint32_t* __restrict__ cell,
                                 float* __restrict__ ox, float* __restrict__ oy, float* __restrict__ oz,
                                 float* __restrict__ vx, float* __restrict__ vy, float* __restrict__ vz,
                                 long long np, float c_kick, double dt, int n,
                                 const long long* __restrict__ pbeg = nullptr,
                                 const long long* __restrict__ pend = nullptr, long long mesh_stride = 0,
                                 int x0 = 0, int nxl = 0, int* __restrict__ err = nullptr) {
    const long long lo = pbeg ? pbeg[blockIdx.y] : 0, hi = pbeg ? pend[blockIdx.y] : np;
    if (pbeg) phi += blockIdx.y * mesh_stride;
    bool outside = false;
    for (long long p = lo + blockIdx.x * (long long)blockDim.x + threadIdx.x; p < hi;
         p += (long long)gridDim.x * blockDim.x) {
        // the particle arrays are touched once per step: streaming (evict-
        // first) loads and stores leave L2 to the potential, which the
        // neighbouring particles re-read
        int i, j, k;
        unpack_cell(__ldcs(cell + p), i, j, k);
        canon_cell<POW2>(i, j, k, n);
        const float tx = __ldcs(ox + p), ty = __ldcs(oy + p), tz = __ldcs(oz + p);
        float gx, gy, gz;
        if constexpr (SLAB) {
            const int li0 = (i & (n - 1)) - x0, li = min(max(li0, 0), nxl - 1);
            outside |= li != li0;
            force_at<ORDER, POW2, true>(phi, n, li + 2, j, k, tx, ty, tz, gx, gy, gz);
            i = li + x0;  // the drift below starts from the (clamped) cell
        } else {
            force_at<ORDER, POW2>(phi, n, i, j, k, tx, ty, tz, gx, gy, gz);
        }
        const float ux = __ldcs(vx + p) + gx * c_kick, uy = __ldcs(vy + p) + gy * c_kick,
                    uz = __ldcs(vz + p) + gz * c_kick;
        __stcs(vx + p, ux);
        __stcs(vy + p, uy);
        __stcs(vz + p, uz);
        if (dt != 0.0) {
            int a, b, c;
            float qa, qb, qc;
            split1((double)i + (double)tx + (double)ux * dt, n, a, qa);
            split1((double)j + (double)ty + (double)uy * dt, n, b, qb);
            split1((double)k + (double)tz + (double)uz * dt, n, c, qc);
            __stcs(cell + p, pack_cell(a, b, c));
            __stcs(ox + p, qa);
            __stcs(oy + p, qb);
            __stcs(oz + p, qc);
        }
    }
    if (SLAB && outside) atomicOr(err, ERRBIT_RANGE);
}

// ---------------------------------------- tiled gather + kick + drift
// The particles in the bin order of the fused deposit (column tile of 4 x 4
// cells, face class, z chunk of 64 cells): one block per super-tile of 2 x 2
// column tiles and one z chunk.  It stages in shared memory the potential
// its particles' stencils reach -- 2 cells below to 2 above the 8 x 8
// columns in x and y (13 x 13 rows), 2 below to 2 above the chunk in z --
// with coalesced loads, then gathers every stencil from there: the neighbour
// particles' re-reads of the potential are served once per block instead of
// once per particle from L1/L2.  Particles are read and written through the
// bin permutation.
constexpr int kGS = 8, kGW = kGS + 5;  // super-tile side in cells; staged rows per axis
constexpr int kGZC = 64, kGZ = kGZC + 5;  // z chunk; staged z values per row
constexpr int kGRL = 72;                  // padded row: z + z / 32 < 72
constexpr size_t kGSmem = (size_t)kGW * kGW * kGRL * sizeof(float);

// Stages work item `item` (super-tile, z chunk) into buffer S: the 13 x 13
// rows by cp.async (one warp per row, every copy in flight, no wait here) and
// the 16 bucket ranges of its particles (rbeg, rlen) by plain loads.
__device__ __forceinline__ void tiles_stage(const float* __restrict__ phi, const uint32_t* __restrict__ off, int n,
                                            int zcb, int item, float* S, uint32_t* rbeg, uint32_t* rlen) {
    const int nt = n >> 2, nst = nt >> 1, m = n - 1;
    const int zc = item & ((1 << zcb) - 1), st = item >> zcb;
    const int sx = st / nst, sy = st - sx * nst;
    const int X0 = sx * kGS, Y0 = sy * kGS, Z0 = zc * kGZC;
    if (threadIdx.x < 16) {  // the 2 x 2 tiles x 4 classes of this chunk
        const int a = threadIdx.x >> 3, b = (threadIdx.x >> 2) & 1, cls = threadIdx.x & 3;
        const uint32_t tile = (uint32_t)(2 * sx + a) * nt + (uint32_t)(2 * sy + b);
        const uint32_t key = ((tile * 4u + cls) << zcb) + (uint32_t)zc;
        const uint32_t beg = __ldg(off + key);
        rbeg[threadIdx.x] = beg;
        rlen[threadIdx.x] = __ldg(off + key + 1) - beg;
    }
    const unsigned pz = (unsigned)n + 2u, plane = (unsigned)n * pz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(S);
    for (int row = warp; row < kGW * kGW; row += 8) {
        const int rx = row / kGW, ry = row - rx * kGW;
        const float* g = phi + (unsigned)((X0 - 2 + rx) & m) * plane + (unsigned)((Y0 - 2 + ry) & m) * pz;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            const int z = lane + 32 * q;
            if (z < kGZ) {
                const uint32_t dst = sbase + (uint32_t)(row * kGRL + z + (z >> 5)) * 4u;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(g + ((Z0 - 2 + z) & m)));
            }
        }
    }
}

// Gathers, kicks and drifts the particles of a staged item.  rpre holds the
// prefix sums of the 16 range lengths.
template <int ORDER>
__device__ __forceinline__ void tiles_compute(const float* S, const uint32_t* rbeg, const uint32_t* rpre, int n,
                                              int zcb, int item, uint32_t* __restrict__ cell, float* __restrict__ ox,
                                              float* __restrict__ oy, float* __restrict__ oz, float* __restrict__ vx,
                                              float* __restrict__ vy, float* __restrict__ vz,
                                              const uint32_t* __restrict__ perm, float c_kick, double dt) {
    const int nst = n >> 3, m = n - 1;
    const int zc = item & ((1 << zcb) - 1), st = item >> zcb;
    const int sx = st / nst, sy = st - sx * nst;
    const int X0 = sx * kGS, Y0 = sy * kGS, Z0 = zc * kGZC;
    const uint32_t total = rpre[16];
    for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
        int r = 0;  // range of t: binary search over the 16 prefix sums
#pragma unroll
        for (int h = 8; h >= 1; h >>= 1)
            if (t >= rpre[r + h]) r += h;
        const uint32_t p = __ldg(perm + rbeg[r] + (t - rpre[r]));
        int i, j, k;
        unpack_cell(__ldcs(cell + p), i, j, k);
        i &= m;
        j &= m;
        k &= m;
        // local coordinates in the staged block (clamped: memory stays in
        // bounds even for a cell word inconsistent with its bucket)
        const int lx = min(max(i - X0 + 2, 2), kGS + 1), ly = min(max(j - Y0 + 2, 2), kGS + 1);
        const int lz = min(max(k - Z0 + 2, 2), kGZC + 1);
        const float tx = __ldcs(ox + p), ty = __ldcs(oy + p), tz = __ldcs(oz + p);
        float gx, gy, gz;
        {
            const SmemStencil<ORDER, kGW, kGRL> sst(S, lx, ly, lz);
            force_from(sst, tx, ty, tz, gx, gy, gz);
        }
        const float ux = __ldcs(vx + p) + gx * c_kick, uy = __ldcs(vy + p) + gy * c_kick,
                    uz = __ldcs(vz + p) + gz * c_kick;
        __stcs(vx + p, ux);
        __stcs(vy + p, uy);
        __stcs(vz + p, uz);
        if (dt != 0.0) {
            int a, b, c;
            float qa, qb, qc;
            split1((double)i + (double)tx + (double)ux * dt, n, a, qa);
            split1((double)j + (double)ty + (double)uy * dt, n, b, qb);
            split1((double)k + (double)tz + (double)uz * dt, n, c, qc);
            __stcs(cell + p, pack_cell(a, b, c));
            __stcs(ox + p, qa);
            __stcs(oy + p, qb);
            __stcs(oz + p, qc);
        }
    }
}

__device__ __forceinline__ void tiles_prefix(uint32_t* rpre, const uint32_t* rlen) {
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        rpre[0] = 0;
        for (int r = 0; r < 16; ++r) rpre[r + 1] = (acc += rlen[r]);
    }
}

// One block per item: stage, wait, compute.
template <int ORDER>
__global__ void __launch_bounds__(256, 4)
k_kick_drift_tiles(const float* __restrict__ phi, uint32_t* __restrict__ cell, float* __restrict__ ox,
                   float* __restrict__ oy, float* __restrict__ oz, float* __restrict__ vx, float* __restrict__ vy,
                   float* __restrict__ vz, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ off, int n,
                   int zcb, float c_kick, double dt) {
    extern __shared__ __align__(16) float S[];
    __shared__ uint32_t rbeg[16], rlen[16], rpre[17];
    tiles_stage(phi, off, n, zcb, (int)blockIdx.x, S, rbeg, rlen);
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    tiles_prefix(rpre, rlen);
    __syncthreads();
    tiles_compute<ORDER>(S, rbeg, rpre, n, zcb, (int)blockIdx.x, cell, ox, oy, oz, vx, vy, vz, perm, c_kick, dt);
}

// ------------------------------------------------ pencil decomposition
// One pencil (x in [x0, x0 + nx), y in [y0, y0 + ny), all z) with its halo
// rows: buffer [nx + 5][ny + 5][n + 2], row (x - x0 + 2, y - y0 + 2), zeroed
// before the deposit (the -1 background is added when the own rows are
// copied out for the z FFT).
// CIC deposit of the pencil's particles into its buffer with shared-nothing
// FP32 atomics: the +1 corners of the last x plane / y row land in the ghost
// rows x = nx (buffer row nx + 2) and y = ny, which the neighbours fold.  A
// cell outside the pencil is recorded in *err and clamped into it.
__global__ void k_pencil_deposit(const uint32_t* __restrict__ cell, const float* __restrict__ ox,
                                 const float* __restrict__ oy, const float* __restrict__ oz, long long np, float mass,
                                 float* __restrict__ buf, int x0, int y0, int nx, int ny, int n, int* err) {
    const long long pz = n + 2, yr = ny + 5;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(__ldg(cell + p), i, j, k);
        int li = (i & (n - 1)) - x0, lj = (j & (n - 1)) - y0;
        k &= n - 1;
        if (li < 0 || li >= nx || lj < 0 || lj >= ny) {
            atomicOr(err, ERRBIT_RANGE);
            li = min(max(li, 0), nx - 1);
            lj = min(max(lj, 0), ny - 1);
        }
        const float fx = __ldg(ox + p), fy = __ldg(oy + p), fz = __ldg(oz + p);
        const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {mass * (1.0f - fz), mass * fz};
        const int kk[2] = {k, (k + 1) & (n - 1)};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                float* row = buf + ((long long)(li + 2 + a) * yr + (lj + 2 + b)) * pz;
                const float w = wx[a] * wy[b];
#pragma unroll
                for (int c = 0; c < 2; ++c) atomicAdd(row + kk[c], w * wz[c]);
            }
    }
}

// Gather + kick + drift of the pencil's particles from its buffer (potential
// with two halo planes / rows below and three above in x and y).
template <int ORDER>
__global__ void __launch_bounds__(256, 3)
k_pencil_kick_drift(const float* __restrict__ buf, uint32_t* __restrict__ cell, float* __restrict__ ox,
                    float* __restrict__ oy, float* __restrict__ oz, float* __restrict__ vx, float* __restrict__ vy,
                    float* __restrict__ vz, long long np, float c_kick, double dt, int n, int x0, int y0, int nx,
                    int ny, int* err) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(__ldcs(cell + p), i, j, k);
        int li = (i & (n - 1)) - x0, lj = (j & (n - 1)) - y0;
        k &= n - 1;
        if (li < 0 || li >= nx || lj < 0 || lj >= ny) {
            atomicOr(err, ERRBIT_RANGE);
            li = min(max(li, 0), nx - 1);
            lj = min(max(lj, 0), ny - 1);
        }
        const float tx = __ldcs(ox + p), ty = __ldcs(oy + p), tz = __ldcs(oz + p);
        float gx, gy, gz;
        {
            const Stencil<ORDER, true, true, true> st(buf, n, li + 2, lj + 2, k, ny + 5);
            force_from(st, tx, ty, tz, gx, gy, gz);
        }
        const float ux = __ldcs(vx + p) + gx * c_kick, uy = __ldcs(vy + p) + gy * c_kick,
                    uz = __ldcs(vz + p) + gz * c_kick;
        __stcs(vx + p, ux);
        __stcs(vy + p, uy);
        __stcs(vz + p, uz);
        if (dt != 0.0) {
            int a, b, c;
            float qa, qb, qc;
            split1((double)(li + x0) + (double)tx + (double)ux * dt, n, a, qa);
            split1((double)(lj + y0) + (double)ty + (double)uy * dt, n, b, qb);
            split1((double)k + (double)tz + (double)uz * dt, n, c, qc);
            __stcs(cell + p, pack_cell(a, b, c));
            __stcs(ox + p, qa);
            __stcs(oy + p, qb);
            __stcs(oz + p, qc);
        }
    }
}

// ----------------------------------------------------- FP32 adjoints
// The FP32 split-position counterparts of csrc/adjoint.cu (same algebra; no
// counterpart in the reference).  With U(c) = scale_d dbar(c) +
// scale_u sum_a u_pa f_a(c), f_a = -G_a phi computed from phi at the corner
// as in force_at, the particle adjoint is xbar_p += sum_c grad W(x_p - c) U(c);
// grad W replaces one factor of the CIC weight by its derivative (-1, +1).
template <int ORDER, bool POW2>
__global__ void __launch_bounds__(256) k_adjoint_gather_f32(
    const uint32_t* __restrict__ cell, const float* __restrict__ ox, const float* __restrict__ oy,
    const float* __restrict__ oz, long long np, const float* __restrict__ dbar, float scale_d,
    const float* __restrict__ phi, const float* __restrict__ ux, const float* __restrict__ uy,
    const float* __restrict__ uz, float scale_u, float* __restrict__ bx, float* __restrict__ by,
    float* __restrict__ bz, int n) {
    const unsigned pz = (unsigned)n + 2u, plane = (unsigned)n * pz;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(__ldg(cell + p), i, j, k);
        canon_cell<POW2>(i, j, k, n);
        const float tx = __ldg(ox + p), ty = __ldg(oy + p), tz = __ldg(oz + p);
        float U[2][2][2] = {};
        if (dbar) {
            const unsigned x0 = (unsigned)wrap_near<POW2>(i, n) * plane, x1 = (unsigned)wrap_near<POW2>(i + 1, n) * plane;
            const unsigned y0 = (unsigned)wrap_near<POW2>(j, n) * pz, y1 = (unsigned)wrap_near<POW2>(j + 1, n) * pz;
            const unsigned z0 = (unsigned)wrap_near<POW2>(k, n), z1 = (unsigned)wrap_near<POW2>(k + 1, n);
            const unsigned xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int c = 0; c < 2; ++c) U[a][b][c] = scale_d * __ldg(dbar + xs[a] + ys[b] + zs[c]);
        }
        if (phi) {
            const float u0 = scale_u * __ldg(ux + p), u1 = scale_u * __ldg(uy + p), u2 = scale_u * __ldg(uz + p);
            const Stencil<ORDER, POW2> st(phi, n, i, j, k);
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        float fx, fy, fz;
                        st.corner(a, b, c, fx, fy, fz);
                        U[a][b][c] += u0 * fx + u1 * fy + u2 * fz;
                    }
        }
        const float w0[2] = {1.0f - tx, tx}, w1[2] = {1.0f - ty, ty}, w2[2] = {1.0f - tz, tz};
        const float dw[2] = {-1.0f, 1.0f};
        float gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    gx += dw[a] * w1[b] * w2[c] * U[a][b][c];
                    gy += w0[a] * dw[b] * w2[c] * U[a][b][c];
                    gz += w0[a] * w1[b] * dw[c] * U[a][b][c];
                }
        bx[p] += gx;
        by[p] += gy;
        bz[p] += gz;
    }
}

// ub_a(c) += sum_p u_pa W(x_p - c) into three unpadded [n][n][n] meshes.
template <bool POW2>
__global__ void k_deposit3_f32(const uint32_t* __restrict__ cell, const float* __restrict__ ox,
                               const float* __restrict__ oy, const float* __restrict__ oz,
                               const float* __restrict__ ux, const float* __restrict__ uy,
                               const float* __restrict__ uz, long long np, float* __restrict__ o0,
                               float* __restrict__ o1, float* __restrict__ o2, int n) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        unpack_cell(__ldg(cell + p), i, j, k);
        canon_cell<POW2>(i, j, k, n);
        const float tx = __ldg(ox + p), ty = __ldg(oy + p), tz = __ldg(oz + p);
        const float w0[2] = {1.0f - tx, tx}, w1[2] = {1.0f - ty, ty}, w2[2] = {1.0f - tz, tz};
        const float u[3] = {__ldg(ux + p), __ldg(uy + p), __ldg(uz + p)};
        const unsigned xs[2] = {(unsigned)wrap_near<POW2>(i, n) * n * n, (unsigned)wrap_near<POW2>(i + 1, n) * n * n};
        const unsigned ys[2] = {(unsigned)wrap_near<POW2>(j, n) * n, (unsigned)wrap_near<POW2>(j + 1, n) * n};
        const unsigned zs[2] = {(unsigned)wrap_near<POW2>(k, n), (unsigned)wrap_near<POW2>(k + 1, n)};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const unsigned o = xs[a] + ys[b] + zs[c];
                    const float w = w0[a] * w1[b] * w2[c];
                    atomicAdd(o0 + o, w * u[0]);
                    atomicAdd(o1 + o, w * u[1]);
                    atomicAdd(o2 + o, w * u[2]);
                }
    }
}

// phibar = -sum_a G_a ub_a on the padded mesh (padding zeroed); G_a the
// 2- or 4-point centred difference of the forward gradient.
template <int ORDER, bool POW2>
__global__ void k_neg_divergence_f32(const float* __restrict__ u0, const float* __restrict__ u1,
                                     const float* __restrict__ u2, float* __restrict__ out, int n) {
    for (long long row = blockIdx.x; row < (long long)n * n; row += gridDim.x) {
        const int i = (int)(row / n), j = (int)(row % n);
        auto R = [&](const float* g, int a, int b) {
            return g + ((long long)wrap_near<POW2>(a, n) * n + wrap_near<POW2>(b, n)) * n;
        };
        const float *xm1 = R(u0, i - 1, j), *xp1 = R(u0, i + 1, j), *xm2 = R(u0, i - 2, j), *xp2 = R(u0, i + 2, j);
        const float *ym1 = R(u1, i, j - 1), *yp1 = R(u1, i, j + 1), *ym2 = R(u1, i, j - 2), *yp2 = R(u1, i, j + 2);
        const float* zc = R(u2, i, j);
        float* o = out + row * (n + 2);
        for (int k = threadIdx.x; k < n + 2; k += blockDim.x) {
            if (k >= n) {
                o[k] = 0.0f;
                continue;
            }
            const int km1 = wrap_near<POW2>(k - 1, n), kp1 = wrap_near<POW2>(k + 1, n);
            const int km2 = wrap_near<POW2>(k - 2, n), kp2 = wrap_near<POW2>(k + 2, n);
            float g;
            if (ORDER == 4)
                g = (8.0f * (xm1[k] - xp1[k]) - (xm2[k] - xp2[k])) * (1.0f / 12.0f) +
                    (8.0f * (ym1[k] - yp1[k]) - (ym2[k] - yp2[k])) * (1.0f / 12.0f) +
                    (8.0f * (zc[km1] - zc[kp1]) - (zc[km2] - zc[kp2])) * (1.0f / 12.0f);
            else
                g = (xm1[k] - xp1[k]) * 0.5f + (ym1[k] - yp1[k]) * 0.5f + (zc[km1] - zc[kp1]) * 0.5f;
            o[k] = -g;
        }
    }
}

__global__ void k_axpy3_f32(float* __restrict__ y0, float* __restrict__ y1, float* __restrict__ y2,
                            const float* __restrict__ x0, const float* __restrict__ x1,
                            const float* __restrict__ x2, float a, long long np) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        y0[p] += a * x0[p];
        y1[p] += a * x1[p];
        y2[p] += a * x2[p];
    }
}

}  // namespace

// ------------------------------------------------------------- launchers
static constexpr int kThreads = 256;

int deposit_f64(const Plan& p, const double* x, const double* y, const double* z, int64_t np,
                double mass, double* mesh) {
    {
        Timed t(p, ST_MESH_INIT);
        k_mesh_init<double><<<grid_for(p, (long long)mesh_elems(p.ng) / 2, kThreads), kThreads, 0, p.stream>>>(mesh, p.ng, -1.0);
    }
    const bool pow2 = (p.ng & (p.ng - 1)) == 0;
    if (np > 0) {
        Timed t(p, ST_DEPOSIT);
        const unsigned g = grid_for(p, np, kThreads);
        if (pow2)
            k_deposit_f64<true><<<g, kThreads, 0, p.stream>>>(x, y, z, np, mass, mesh, p.ng, p.d_err);
        else
            k_deposit_f64<false><<<g, kThreads, 0, p.stream>>>(x, y, z, np, mass, mesh, p.ng, p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int gradient_f64(const Plan& p, const double* phi, double* fx, double* fy, double* fz) {
    const bool pow2 = (p.ng & (p.ng - 1)) == 0;
    const unsigned g = grid_for(p, (long long)p.ng * p.ng, 1);
    {
        Timed t(p, ST_GRADIENT);
        if (p.grad_order == 4 && pow2)
            k_gradient_f64<4, true><<<g, kThreads, 0, p.stream>>>(phi, fx, fy, fz, p.ng);
        else if (p.grad_order == 4)
            k_gradient_f64<4, false><<<g, kThreads, 0, p.stream>>>(phi, fx, fy, fz, p.ng);
        else if (pow2)
            k_gradient_f64<2, true><<<g, kThreads, 0, p.stream>>>(phi, fx, fy, fz, p.ng);
        else
            k_gradient_f64<2, false><<<g, kThreads, 0, p.stream>>>(phi, fx, fy, fz, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int interp_kick_f64(const Plan& p, const double* x, const double* y, const double* z,
                    const double* fx, const double* fy, const double* fz, double* px, double* py,
                    double* pz, int64_t np, double c_kick) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_INTERP_KICK);
        const unsigned g = grid_for(p, np, kThreads);
        if ((p.ng & (p.ng - 1)) == 0)
            k_interp_kick_f64<true><<<g, kThreads, 0, p.stream>>>(x, y, z, fx, fy, fz, px, py, pz, np, c_kick, p.ng,
                                                                  p.d_err);
        else
            k_interp_kick_f64<false><<<g, kThreads, 0, p.stream>>>(x, y, z, fx, fy, fz, px, py, pz, np, c_kick, p.ng,
                                                                   p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int drift_f64(const Plan& p, double* x, double* y, double* z, const double* px, const double* py,
              const double* pz, int64_t np, double dt) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_DRIFT);
        k_drift_f64<<<grid_for(p, np, kThreads), kThreads, 0, p.stream>>>(x, y, z, px, py, pz, np, dt, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int split_positions(const Plan& p, const double* x, const double* y, const double* z, int64_t np,
                    uint32_t* cell, float* ox, float* oy, float* oz) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_SPLIT);
        k_split<<<grid_for(p, np, kThreads), kThreads, 0, p.stream>>>(x, y, z, np, cell, ox, oy, oz, p.ng, p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int join_positions(const Plan& p, const uint32_t* cell, const float* ox, const float* oy,
                   const float* oz, int64_t np, double* x, double* y, double* z) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_SPLIT);
        k_join<<<grid_for(p, np, kThreads), kThreads, 0, p.stream>>>(cell, ox, oy, oz, np, x, y, z);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int interp_f32(const Plan& p, const float* phi, const uint32_t* cell, const float* ox,
               const float* oy, const float* oz, int64_t np, float* fx, float* fy, float* fz) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_INTERP);
        const unsigned g = grid_for(p, np, kThreads);
        const bool pow2 = (p.ng & (p.ng - 1)) == 0;
        if (p.grad_order == 4 && pow2)
            k_interp_f32<4, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, np, fx, fy, fz, p.ng);
        else if (p.grad_order == 4)
            k_interp_f32<4, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, np, fx, fy, fz, p.ng);
        else if (pow2)
            k_interp_f32<2, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, np, fx, fy, fz, p.ng);
        else
            k_interp_f32<2, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, np, fx, fy, fz, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int kick_drift_f32(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz,
                   float* vx, float* vy, float* vz, int64_t np, double c_kick, double dt) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_KICK_DRIFT);
        const unsigned g = grid_for(p, np, kThreads);
        const bool pow2 = (p.ng & (p.ng - 1)) == 0;
        const float ck = (float)c_kick;
        if (p.grad_order == 4 && pow2)
            k_kick_drift_f32<4, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck, dt, p.ng);
        else if (p.grad_order == 4)
            k_kick_drift_f32<4, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck, dt, p.ng);
        else if (pow2)
            k_kick_drift_f32<2, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck, dt, p.ng);
        else
            k_kick_drift_f32<2, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck, dt, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// Gather + kick + drift of the particles of one x-slab; phi is the slab's
// buffer (plane 0 = x0 - 2).  Power-of-two meshes only.
int slab_kick_drift_f32(const Plan& p, int x0, int nx, const float* phi, uint32_t* cell, float* ox, float* oy,
                        float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick, double dt) {
    if (np == 0) return PM_OK;
    const unsigned g = grid_for(p, np, kThreads, 4);
    const float ck = (float)c_kick;
    {
        Timed t(p, ST_KICK_DRIFT);
        if (p.grad_order == 4)
            k_kick_drift_f32<4, true, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck,
                                                                          dt, p.ng, nullptr, nullptr, 0, x0, nx,
                                                                          p.d_err);
        else
            k_kick_drift_f32<2, true, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np, ck,
                                                                          dt, p.ng, nullptr, nullptr, 0, x0, nx,
                                                                          p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_deposit_f32(const Plan& p, int x0, int y0, int nx, int ny, const uint32_t* cell, const float* ox,
                       const float* oy, const float* oz, int64_t np, float mass, float* buf) {
    PMB_CUDA_CHECK(cudaMemsetAsync(buf, 0, (size_t)(nx + 5) * (ny + 5) * (p.ng + 2) * sizeof(float), p.stream));
    if (np > 0) {
        Timed t(p, ST_DEPOSIT);
        k_pencil_deposit<<<grid_for(p, np, kThreads, 8), kThreads, 0, p.stream>>>(cell, ox, oy, oz, np, mass, buf, x0,
                                                                                  y0, nx, ny, p.ng, p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pencil_kick_drift_f32(const Plan& p, int x0, int y0, int nx, int ny, const float* buf, uint32_t* cell, float* ox,
                          float* oy, float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick,
                          double dt) {
    if (np == 0) return PM_OK;
    const unsigned g = grid_for(p, np, kThreads, 3);
    {
        Timed t(p, ST_KICK_DRIFT);
        if (p.grad_order == 4)
            k_pencil_kick_drift<4><<<g, kThreads, 0, p.stream>>>(buf, cell, ox, oy, oz, vx, vy, vz, np, (float)c_kick,
                                                                 dt, p.ng, x0, y0, nx, ny, p.d_err);
        else
            k_pencil_kick_drift<2><<<g, kThreads, 0, p.stream>>>(buf, cell, ox, oy, oz, vx, vy, vz, np, (float)c_kick,
                                                                 dt, p.ng, x0, y0, nx, ny, p.d_err);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

bool tiled_gather_supported(int ng) { return ng >= 256 && ng <= 1024 && (ng & (ng - 1)) == 0; }

int tiled_gather_zcb(int ng) {
    int b = 0;
    while ((kGZC << b) < ng) ++b;
    return b;
}

// One-time kernel attribute (48.7 KB of dynamic shared memory), set on the
// plan's device when an FP32 plan is created.
int tiled_gather_prepare() {
    PMB_CUDA_CHECK(cudaFuncSetAttribute(k_kick_drift_tiles<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGSmem));
    PMB_CUDA_CHECK(cudaFuncSetAttribute(k_kick_drift_tiles<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGSmem));
    return PM_OK;
}

int kick_drift_tiles_f32(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                         float* vy, float* vz, int64_t np, double c_kick, double dt) {
    if (np == 0) return PM_OK;
    if (!tiled_gather_supported(p.ng)) return fail(PM_ERR_SIZE, "tiled gather needs a power-of-two ng in [256, 1024]");
    const int zcb = tiled_gather_zcb(p.ng);
    const int items = ((p.ng / kGS) * (p.ng / kGS)) << zcb;
    const float ck = (float)c_kick;
    {
        Timed t(p, ST_KICK_DRIFT);
        if (p.grad_order == 4) {
            k_kick_drift_tiles<4><<<(unsigned)items, 256, kGSmem, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz,
                                                                              p.tiles.perm, p.tiles.off, p.ng, zcb, ck,
                                                                              dt);
        } else {
            k_kick_drift_tiles<2><<<(unsigned)items, 256, kGSmem, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz,
                                                                              p.tiles.perm, p.tiles.off, p.ng, zcb, ck,
                                                                              dt);
        }
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// ------------------------------------------------------- FP32 adjoints
int adjoint_gather_f32(const Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                       int64_t np, const float* dbar, double scale_d, const float* phi, const float* u[3],
                       double scale_u, float* xbar[3]) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_ADJOINT);
        const unsigned g = grid_for(p, np, kThreads);
        const bool pow2 = (p.ng & (p.ng - 1)) == 0;
        const float* u0 = u ? u[0] : nullptr;
        const float* u1 = u ? u[1] : nullptr;
        const float* u2 = u ? u[2] : nullptr;
#define PMB_ADJ_G(O, P2)                                                                                   \
    k_adjoint_gather_f32<O, P2><<<g, kThreads, 0, p.stream>>>(cell, ox, oy, oz, np, dbar, (float)scale_d, phi, \
                                                              u0, u1, u2, (float)scale_u, xbar[0], xbar[1],  \
                                                              xbar[2], p.ng)
        if (p.grad_order == 4 && pow2) PMB_ADJ_G(4, true);
        else if (p.grad_order == 4) PMB_ADJ_G(4, false);
        else if (pow2) PMB_ADJ_G(2, true);
        else PMB_ADJ_G(2, false);
#undef PMB_ADJ_G
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int adjoint_mesh_source_f32(const Plan& p, const uint32_t* cell, const float* ox, const float* oy,
                            const float* oz, const float* u[3], int64_t np, float* ub[3], float* phibar) {
    const size_t cells = (size_t)p.ng * p.ng * p.ng;
    for (int a = 0; a < 3; ++a) PMB_CUDA_CHECK(cudaMemsetAsync(ub[a], 0, cells * sizeof(float), p.stream));
    {
        Timed t(p, ST_ADJOINT, 2);
        const bool pow2 = (p.ng & (p.ng - 1)) == 0;
        if (np > 0) {
            const unsigned g = grid_for(p, np, kThreads);
            if (pow2)
                k_deposit3_f32<true><<<g, kThreads, 0, p.stream>>>(cell, ox, oy, oz, u[0], u[1], u[2], np, ub[0],
                                                                    ub[1], ub[2], p.ng);
            else
                k_deposit3_f32<false><<<g, kThreads, 0, p.stream>>>(cell, ox, oy, oz, u[0], u[1], u[2], np, ub[0],
                                                                     ub[1], ub[2], p.ng);
        }
        const unsigned gr = grid_for(p, (long long)p.ng * p.ng, 1);
        if (p.grad_order == 4 && pow2)
            k_neg_divergence_f32<4, true><<<gr, kThreads, 0, p.stream>>>(ub[0], ub[1], ub[2], phibar, p.ng);
        else if (p.grad_order == 4)
            k_neg_divergence_f32<4, false><<<gr, kThreads, 0, p.stream>>>(ub[0], ub[1], ub[2], phibar, p.ng);
        else if (pow2)
            k_neg_divergence_f32<2, true><<<gr, kThreads, 0, p.stream>>>(ub[0], ub[1], ub[2], phibar, p.ng);
        else
            k_neg_divergence_f32<2, false><<<gr, kThreads, 0, p.stream>>>(ub[0], ub[1], ub[2], phibar, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int axpy3_f32(const Plan& p, float* y[3], const float* x[3], double a, int64_t np) {
    if (np == 0) return PM_OK;
    k_axpy3_f32<<<grid_for(p, np, kThreads), kThreads, 0, p.stream>>>(y[0], y[1], y[2], x[0], x[1], x[2], (float)a,
                                                                       np);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

}  // namespace pmb

namespace pmb {

int kick_drift_f32_batch(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz,
                         float* vx, float* vy, float* vz, const long long* pbeg, const long long* pend, int nbox,
                         int64_t np_total, double c_kick, double dt) {
    if (np_total == 0) return PM_OK;
    const long long per_box = (np_total + nbox - 1) / nbox;
    dim3 g(grid_for(p, per_box, kThreads, 2), nbox);
    const long long ms = (long long)mesh_elems(p.ng);
    {
        Timed t(p, ST_KICK_DRIFT);
        const bool pow2 = (p.ng & (p.ng - 1)) == 0;
        const float ck = (float)c_kick;
        if (p.grad_order == 4 && pow2)
            k_kick_drift_f32<4, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np_total, ck,
                                                                  dt, p.ng, pbeg, pend, ms);
        else if (p.grad_order == 4)
            k_kick_drift_f32<4, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np_total, ck,
                                                                   dt, p.ng, pbeg, pend, ms);
        else if (pow2)
            k_kick_drift_f32<2, true><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np_total, ck,
                                                                  dt, p.ng, pbeg, pend, ms);
        else
            k_kick_drift_f32<2, false><<<g, kThreads, 0, p.stream>>>(phi, cell, ox, oy, oz, vx, vy, vz, np_total, ck,
                                                                   dt, p.ng, pbeg, pend, ms);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

}  // namespace pmb
