/*
 * pm_oracle.c -- CPU FP64 restatement of the reference particle-mesh step.
 *
 * TEST INFRASTRUCTURE, NOT PRODUCT.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker.
 * The CUDA path never calls into it.
 *
 * Single box, one rank, periodic.  The reference splits the mesh over MPI
 * ranks with +1 ghost planes (deposit) and -1/+2 ghost planes (gradient); on
 * one box every ghost is the periodic image, so each ghost access below is a
 * periodic index wrap.  Each function names the reference lines it restates.
 *
 * Layouts (all row-major, z fastest):
 *   mesh    real   [ng][ng][ng+2]   (the FFTW in-place stride, src/core/main.cpp:24-28)
 *   spectrum cplx  [ng][ng][ng/2+1] (same bytes, x = kx, y = ky, z = kz)
 *   force   real   [ng][ng][ng]     (one array per component)
 *   particles      SoA double x[], y[], z[] in cell units, [0, ng)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define PADZ(ng) ((long)(ng) + 2)

static inline long wrapl(long i, long n) {
    long r = i % n;
    return r < 0 ? r + n : r;
}

/* ---------------------------------------------------------------- deposit */

/* CIC deposit of the density contrast delta = -1 + sum_p m W(x_p - c).
 *   init_buf       src/utils/utils.cpp:38-68        (owned cells start at -1)
 *   deposit        src/utils/utils.cpp:70-102       (cell = int(x), t = x - cell)
 *   cic_deposit    include/utils/utils_inline.h:25-49 (weights (1-t, t) on i, i+1)
 *   ghost fold     src/decomp/slab/transpose_slab.cpp:23-27 and
 *                  src/decomp/slab/reorder_slab.cpp:13-18 (ghost planes summed
 *                  into the periodic image) -> here i+1 wraps to 0.
 * Pad cells z = ng, ng+1 are set to 0. */
void orc_deposit(int ng, long np, const double* x, const double* y, const double* z, double mass,
                 double* mesh) {
    const long pz = PADZ(ng);
    for (long i = 0; i < ng; ++i)
        for (long j = 0; j < ng; ++j) {
            double* row = mesh + (i * ng + j) * pz;
            for (long k = 0; k < ng; ++k) row[k] = -1.0;
            row[ng] = 0.0;
            row[ng + 1] = 0.0;
        }
    for (long p = 0; p < np; ++p) {
        const double fx = floor(x[p]), fy = floor(y[p]), fz = floor(z[p]);
        const double tx = x[p] - fx, ty = y[p] - fy, tz = z[p] - fz;
        const long i0 = wrapl((long)fx, ng), j0 = wrapl((long)fy, ng), k0 = wrapl((long)fz, ng);
        const long i1 = (i0 + 1) % ng, j1 = (j0 + 1) % ng, k1 = (k0 + 1) % ng;
        const double sx0 = 1.0 - tx, sy0 = 1.0 - ty, sz0 = 1.0 - tz;
        const double sxy00 = sx0 * sy0, sxy10 = tx * sy0, sxy01 = sx0 * ty, sxy11 = tx * ty;
        const double m0 = mass * sz0, m1 = mass * tz;
        mesh[(i0 * ng + j0) * pz + k0] += sxy00 * m0;
        mesh[(i1 * ng + j0) * pz + k0] += sxy10 * m0;
        mesh[(i0 * ng + j1) * pz + k0] += sxy01 * m0;
        mesh[(i1 * ng + j1) * pz + k0] += sxy11 * m0;
        mesh[(i0 * ng + j0) * pz + k1] += sxy00 * m1;
        mesh[(i1 * ng + j0) * pz + k1] += sxy10 * m1;
        mesh[(i0 * ng + j1) * pz + k1] += sxy01 * m1;
        mesh[(i1 * ng + j1) * pz + k1] += sxy11 * m1;
    }
}

/* -------------------------------------------------------------------- FFT */

/* Mixed-radix complex DFT, unnormalised, X[k] = sum_n x[n] e^{sign 2 pi i nk/n}.
 * Radices are taken in FFTE's preference order 8, 5, 4, 3, 2
 * (src/fft/ffte1/factor.f:19-43; twiddles W = exp(-2 pi i jk/n),
 * src/fft/ffte1/fft235.f:205-219).  Recursive decimation in time; any n whose
 * factors are 2, 3, 5 is supported (others fall back to a direct DFT). */
static void twiddle(long num, long den, int sign, double* c, double* s) {
    long r = wrapl(num, den);
    long double ang = (long double)sign * 2.0L * 3.141592653589793238462643383279502884L *
                      (long double)r / (long double)den;
    *c = (double)cosl(ang);
    *s = (double)sinl(ang);
}

static int pick_radix(long n) {
    if (n % 8 == 0 && n != 16) return 8;
    if (n % 5 == 0) return 5;
    if (n % 4 == 0) return 4;
    if (n % 3 == 0) return 3;
    if (n % 2 == 0) return 2;
    return (int)n;
}

/* in: n complex values at stride `is` (complex units); out: n contiguous. */
static void fft_rec(long n, const double* in, long is, double* out, int sign, double* work) {
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    const int r = pick_radix(n);
    const long m = n / r;
    if (m == 1) { /* direct DFT of length r */
        for (long k = 0; k < n; ++k) {
            double re = 0, im = 0;
            for (long q = 0; q < n; ++q) {
                double c, s;
                twiddle(q * k, n, sign, &c, &s);
                const double a = in[2 * q * is], b = in[2 * q * is + 1];
                re += a * c - b * s;
                im += a * s + b * c;
            }
            out[2 * k] = re;
            out[2 * k + 1] = im;
        }
        return;
    }
    /* sub-transforms of the r decimated sequences into work[q*m + k] */
    for (int q = 0; q < r; ++q) fft_rec(m, in + 2 * q * is, is * r, work + 2 * q * m, sign, out);
    for (long k = 0; k < m; ++k)
        for (int s = 0; s < r; ++s) {
            const long kk = k + s * m;
            double re = 0, im = 0;
            for (int q = 0; q < r; ++q) {
                double c, sn;
                twiddle((long)q * kk, n, sign, &c, &sn);
                const double a = work[2 * (q * m + k)], b = work[2 * (q * m + k) + 1];
                re += a * c - b * sn;
                im += a * sn + b * c;
            }
            out[2 * kk] = re;
            out[2 * kk + 1] = im;
        }
}

/* 1D complex FFT, in place on n interleaved complex values at stride `stride`. */
void orc_fft1d(long n, double* data, long stride, int sign) {
    double* in = (double*)malloc(sizeof(double) * 2 * n);
    double* out = (double*)malloc(sizeof(double) * 2 * n);
    double* work = (double*)malloc(sizeof(double) * 2 * n);
    for (long i = 0; i < n; ++i) {
        in[2 * i] = data[2 * i * stride];
        in[2 * i + 1] = data[2 * i * stride + 1];
    }
    /* each recursion level alternates `out` and `work` as its scratch */
    fft_rec(n, in, 1, out, sign, work);
    for (long i = 0; i < n; ++i) {
        data[2 * i * stride] = out[2 * i];
        data[2 * i * stride + 1] = out[2 * i + 1];
    }
    free(in);
    free(out);
    free(work);
}

/* In-place unnormalised R2C of mesh [ng][ng][ng+2] -> spectrum [kx][ky][kz].
 * Restates FFT::forward, src/fft/fftw/fft.cpp:96 (fftw_mpi r2c, sign -1;
 * FFTE: src/fft/ffte1/pdzfft3d.f:77-264).  The spectrum is left in natural
 * [kx][ky][kz] order; the reference's TRANSPOSED_OUT order only swaps kx and
 * ky and every later stage here is symmetric in them. */
void orc_rfft3d_forward(int ng, double* mesh) {
    const long n = ng, h = ng / 2 + 1, pz = PADZ(ng);
    double* line = (double*)malloc(sizeof(double) * 2 * n);
    for (long i = 0; i < n; ++i)
        for (long j = 0; j < n; ++j) {
            double* row = mesh + (i * n + j) * pz;
            for (long k = 0; k < n; ++k) {
                line[2 * k] = row[k];
                line[2 * k + 1] = 0.0;
            }
            orc_fft1d(n, line, 1, -1);
            for (long k = 0; k < h; ++k) {
                row[2 * k] = line[2 * k];
                row[2 * k + 1] = line[2 * k + 1];
            }
        }
    free(line);
    double* c = mesh; /* complex view, element (x,y,kz) at 2*((x*n + y)*h + kz) */
    for (long i = 0; i < n; ++i)
        for (long k = 0; k < h; ++k) orc_fft1d(n, c + 2 * (i * n * h + k), h, -1);
    for (long j = 0; j < n; ++j)
        for (long k = 0; k < h; ++k) orc_fft1d(n, c + 2 * (j * h + k), n * h, -1);
}

/* In-place unnormalised C2R, the inverse of orc_rfft3d_forward up to a factor
 * ng^3.  Restates FFT::backward, src/fft/fftw/fft.cpp:97 (FFTW c2r: the
 * imaginary parts of the kz = 0 and kz = ng/2 entries are ignored). */
void orc_rfft3d_inverse(int ng, double* mesh) {
    const long n = ng, h = ng / 2 + 1, pz = PADZ(ng);
    double* c = mesh;
    for (long j = 0; j < n; ++j)
        for (long k = 0; k < h; ++k) orc_fft1d(n, c + 2 * (j * h + k), n * h, +1);
    for (long i = 0; i < n; ++i)
        for (long k = 0; k < h; ++k) orc_fft1d(n, c + 2 * (i * n * h + k), h, +1);
    double* line = (double*)malloc(sizeof(double) * 2 * n);
    for (long i = 0; i < n; ++i)
        for (long j = 0; j < n; ++j) {
            double* row = mesh + (i * n + j) * pz;
            for (long k = 0; k < h; ++k) {
                line[2 * k] = row[2 * k];
                line[2 * k + 1] = row[2 * k + 1];
            }
            line[1] = 0.0;
            line[2 * (n / 2) + 1] = 0.0;
            for (long k = h; k < n; ++k) {
                line[2 * k] = line[2 * (n - k)];
                line[2 * k + 1] = -line[2 * (n - k) + 1];
            }
            orc_fft1d(n, line, 1, +1);
            for (long k = 0; k < n; ++k) row[k] = line[2 * k];
            row[n] = 0.0;
            row[n + 1] = 0.0;
        }
    free(line);
}

/* ------------------------------------------------------------------ Green */

/* phi_hat = delta_hat * G.
 * kind 0 (reference): G = -c / (2 N^3 (3 - cos 2pi i/N - cos 2pi j/N - cos 2pi k/N)),
 *   the inverse 7-point Laplacian times c.  With c = 3 Omega_0 / (2a) this is
 *   the reference table times 1/a: src/fft/fftw/fft.cpp:50-57 and :75-82.
 * kind 1 (spectral): G = -c / (N^3 |k|^2), k = 2 pi m / N with m the signed
 *   frequency (new; the reference has the discrete kernel only).
 * G(0) = 0 in both (fft.cpp:56). */
void orc_green(int ng, double* spec, double c, int kind) {
    const long n = ng, h = ng / 2 + 1;
    const double n3 = (double)n * (double)n * (double)n;
    const long double twopi_n = 2.0L * 3.141592653589793238462643383279502884L / (long double)n;
    for (long i = 0; i < n; ++i)
        for (long j = 0; j < n; ++j)
            for (long k = 0; k < h; ++k) {
                double* v = spec + 2 * ((i * n + j) * h + k);
                double g;
                if (i == 0 && j == 0 && k == 0) {
                    g = 0.0;
                } else if (kind == 0) {
                    const double s = 3.0 - (double)cosl(twopi_n * i) - (double)cosl(twopi_n * j) -
                                     (double)cosl(twopi_n * k);
                    g = -c / (2.0 * n3 * s);
                } else {
                    const long mi = i <= n / 2 ? i : i - n, mj = j <= n / 2 ? j : j - n;
                    const double k2 = (double)(twopi_n * twopi_n) * (double)(mi * mi + mj * mj + k * k);
                    g = -c / (n3 * k2);
                }
                v[0] *= g;
                v[1] *= g;
            }
}

/* --------------------------------------------------------------- gradient */

/* f = -grad(phi) on the periodic mesh.  phi is the padded real mesh
 * [ng][ng][ng+2]; f* are [ng][ng][ng].
 * order 2 (reference): f = (phi[i-1] - phi[i+1]) / 2, src/utils/utils.cpp:115-137
 *   with the -1/+2 ghost planes of src/decomp/slab/reorder_slab_back.cpp:13-34
 *   and transpose_slab_back.cpp:3-45 replaced by periodic wraps.
 * order 4 (new): f = (8(phi[i-1] - phi[i+1]) - (phi[i-2] - phi[i+2])) / 12. */
void orc_gradient(int ng, int order, const double* phi, double* fx, double* fy, double* fz) {
    const long n = ng, pz = PADZ(ng);
#define PHI(a, b, c) phi[(wrapl((a), n) * n + wrapl((b), n)) * pz + wrapl((c), n)]
    for (long i = 0; i < n; ++i)
        for (long j = 0; j < n; ++j)
            for (long k = 0; k < n; ++k) {
                const long o = (i * n + j) * n + k;
                if (order == 4) {
                    fx[o] = (8.0 * (PHI(i - 1, j, k) - PHI(i + 1, j, k)) - (PHI(i - 2, j, k) - PHI(i + 2, j, k))) / 12.0;
                    fy[o] = (8.0 * (PHI(i, j - 1, k) - PHI(i, j + 1, k)) - (PHI(i, j - 2, k) - PHI(i, j + 2, k))) / 12.0;
                    fz[o] = (8.0 * (PHI(i, j, k - 1) - PHI(i, j, k + 1)) - (PHI(i, j, k - 2) - PHI(i, j, k + 2))) / 12.0;
                } else {
                    fx[o] = (PHI(i - 1, j, k) - PHI(i + 1, j, k)) * 0.5;
                    fy[o] = (PHI(i, j - 1, k) - PHI(i, j + 1, k)) * 0.5;
                    fz[o] = (PHI(i, j, k - 1) - PHI(i, j, k + 1)) * 0.5;
                }
            }
#undef PHI
}

/* ------------------------------------------------------ interpolate + kick */

/* Trilinear (CIC) gather of a [ng][ng][ng] mesh at a particle, periodic.
 * Same operation order as trilerp1, include/utils/utils_inline.h:55-70. */
static inline double trilerp(const double* f, long n, long i0, long j0, long k0, double tx,
                             double ty, double tz) {
    const long i1 = (i0 + 1) % n, j1 = (j0 + 1) % n, k1 = (k0 + 1) % n;
    const double mx = 1.0 - tx, my = 1.0 - ty, mz = 1.0 - tz;
#define F(a, b, c) f[((a) * n + (b)) * n + (c)]
    const double f00 = F(i0, j0, k0) * mx + F(i1, j0, k0) * tx;
    const double f10 = F(i0, j1, k0) * mx + F(i1, j1, k0) * tx;
    const double fz0 = f00 * my + f10 * ty;
    const double g00 = F(i0, j0, k1) * mx + F(i1, j0, k1) * tx;
    const double g10 = F(i0, j1, k1) * mx + F(i1, j1, k1) * tx;
    const double fz1 = g00 * my + g10 * ty;
#undef F
    return fz0 * mz + fz1 * tz;
}

/* p += c_kick * W^T f at each particle.  src/utils/utils.cpp:141-170; the
 * reference's c_kick is Da * function_a(a) (utils.cpp:142,
 * include/utils/utils_inline.h:51-53). */
void orc_interp_kick(int ng, long np, const double* x, const double* y, const double* z,
                     const double* fx, const double* fy, const double* fz, double* px, double* py,
                     double* pz, double c_kick) {
    const long n = ng;
    for (long p = 0; p < np; ++p) {
        const double flx = floor(x[p]), fly = floor(y[p]), flz = floor(z[p]);
        const double tx = x[p] - flx, ty = y[p] - fly, tz = z[p] - flz;
        const long i0 = wrapl((long)flx, n), j0 = wrapl((long)fly, n), k0 = wrapl((long)flz, n);
        px[p] += trilerp(fx, n, i0, j0, k0, tx, ty, tz) * c_kick;
        py[p] += trilerp(fy, n, i0, j0, k0, tx, ty, tz) * c_kick;
        pz[p] += trilerp(fz, n, i0, j0, k0, tx, ty, tz) * c_kick;
    }
}

/* x += dt * p, wrapped into [0, ng).  New: the reference never moves
 * particles (src/core/main.cpp:90-139). */
static inline double wrap_pos(double v, double n) {
    v = v - n * floor(v / n);
    return v >= n ? v - n : v; /* v/n rounding can land exactly on n */
}
void orc_drift(int ng, long np, double* x, double* y, double* z, const double* px,
               const double* py, const double* pz, double dt) {
    const double n = (double)ng;
    for (long p = 0; p < np; ++p) {
        x[p] = wrap_pos(x[p] + px[p] * dt, n);
        y[p] = wrap_pos(y[p] + py[p] * dt, n);
        z[p] = wrap_pos(z[p] + pz[p] * dt, n);
    }
}
