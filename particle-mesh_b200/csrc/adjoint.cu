// Adjoint (vector-Jacobian) kernels of the particle-mesh step, FP64.
//
// No counterpart in the reference, which has no differentiation.  The force
// on particle p is F_p(x) = sum_c W(x_p - c) f(c) with f_a = G_a phi,
// phi = P delta, delta = -1 + m sum_q W(x_q - c): W the CIC weight, G_a the
// centred difference (antisymmetric on the periodic mesh, G_a^T = -G_a), P
// the Green's-function Poisson operator (a real, even Fourier multiplier,
// hence symmetric).  For adjoint particle vectors u (one 3-vector per
// particle) the vector-Jacobian product is
//
//   (dF/dx)^T u |_p = sum_a u_pa grad W(x_p - c) . f_a(c)            (direct)
//                   + m grad W(x_p - c) . P( -sum_a G_a D_a(u) )(c)   (mesh)
//
// with D_a(u)(c) = sum_q u_qa W(x_q - c) the CIC deposit of u's component a
// (the transpose of interpolation).  grad W is piecewise constant: along x,
// d/dx of the weights (1 - t, t) on cells (i0, i0+1) is (-1, +1).  The same
// gather gives the adjoint of the density deposit itself:
// d delta / d x_p ^T dbar = m grad W(x_p - c) . dbar(c).
#include "pm_internal.cuh"

namespace pmb {

namespace {

// Neighbour index c in [-n, 2n) wrapped into [0, n) (any mesh size).
__device__ __forceinline__ int wrp(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

__device__ __forceinline__ double wrapped(double v, double n) {
    if (v >= 0.0 && v < n) return v;
    double m = v - n * floor(v / n);
    return m >= n ? m - n : (m < 0.0 ? 0.0 : m);
}

// ub_a(c) = sum_p u_pa W(x_p - c), three unpadded [n][n][n] meshes (zeroed
// by the caller); FP64 atomics.
__global__ void k_deposit3_f64(const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ ux,
                               const double* __restrict__ uy, const double* __restrict__ uz, long long np,
                               double* __restrict__ ox, double* __restrict__ oy, double* __restrict__ oz, int n) {
    const double dn = (double)n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        const double xp = wrapped(x[p], dn), yp = wrapped(y[p], dn), zp = wrapped(z[p], dn);
        const double fx = floor(xp), fy = floor(yp), fz = floor(zp);
        const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
        const double tx = xp - fx, ty = yp - fy, tz = zp - fz;
        const double wx[2] = {1.0 - tx, tx}, wy[2] = {1.0 - ty, ty}, wz[2] = {1.0 - tz, tz};
        const double u[3] = {ux[p], uy[p], uz[p]};
        double* out[3] = {ox, oy, oz};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const long long o = ((long long)wrp(i0 + a, n) * n + wrp(j0 + b, n)) * n + wrp(k0 + c, n);
                    const double w = wx[a] * wy[b] * wz[c];
#pragma unroll
                    for (int d = 0; d < 3; ++d) atomicAdd(out[d] + o, w * u[d]);
                }
    }
}

// phibar = -sum_a G_a ub_a on the padded mesh [n][n][n+2] (padding zeroed),
// G_a the plan's centred difference: G_a g(c) = (g(c - e_a) - g(c + e_a)) / 2
// (2-point) or (8 (g(c-e) - g(c+e)) - (g(c-2e) - g(c+2e))) / 12 (4-point).
template <int ORDER>
__global__ void k_neg_divergence_f64(const double* __restrict__ ux, const double* __restrict__ uy,
                                     const double* __restrict__ uz, double* __restrict__ phibar, int n) {
    const long long pz = n + 2;
    for (long long row = blockIdx.x; row < (long long)n * n; row += gridDim.x) {
        const int i = (int)(row / n), j = (int)(row % n);
        auto R = [&](const double* g, int a, int b) { return g + ((long long)wrp(a, n) * n + wrp(b, n)) * n; };
        const double *xm1 = R(ux, i - 1, j), *xp1 = R(ux, i + 1, j), *xm2 = R(ux, i - 2, j), *xp2 = R(ux, i + 2, j);
        const double *ym1 = R(uy, i, j - 1), *yp1 = R(uy, i, j + 1), *ym2 = R(uy, i, j - 2), *yp2 = R(uy, i, j + 2);
        const double* zc = R(uz, i, j);
        double* out = phibar + row * pz;
        for (int k = threadIdx.x; k < n + 2; k += blockDim.x) {
            if (k >= n) {
                out[k] = 0.0;
                continue;
            }
            const int km1 = wrp(k - 1, n), kp1 = wrp(k + 1, n), km2 = wrp(k - 2, n), kp2 = wrp(k + 2, n);
            double g;
            if (ORDER == 4)
                g = (8.0 * (xm1[k] - xp1[k]) - (xm2[k] - xp2[k])) / 12.0 +
                    (8.0 * (ym1[k] - yp1[k]) - (ym2[k] - yp2[k])) / 12.0 +
                    (8.0 * (zc[km1] - zc[kp1]) - (zc[km2] - zc[kp2])) / 12.0;
            else
                g = (xm1[k] - xp1[k]) * 0.5 + (ym1[k] - yp1[k]) * 0.5 + (zc[km1] - zc[kp1]) * 0.5;
            out[k] = -g;
        }
    }
}

// grad of sum_c W(x_p - c) g(c) with respect to x_p, g unpadded (stride n)
// or padded (stride n + 2).
__device__ __forceinline__ void grad_gather(const double* __restrict__ g, long long pz, int n, int i0, int j0,
                                            int k0, double tx, double ty, double tz, double& gx, double& gy,
                                            double& gz) {
    const double wx[2] = {1.0 - tx, tx}, wy[2] = {1.0 - ty, ty}, wz[2] = {1.0 - tz, tz};
    const double dw[2] = {-1.0, 1.0};
    gx = gy = gz = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const double v = __ldg(g + ((long long)wrp(i0 + a, n) * n + wrp(j0 + b, n)) * pz + wrp(k0 + c, n));
                gx += dw[a] * wy[b] * wz[c] * v;
                gy += wx[a] * dw[b] * wz[c] * v;
                gz += wx[a] * wy[b] * dw[c] * v;
            }
}

// xbar_p += scale_d * m * grad W . dbar  +  scale_u * sum_a u_pa grad W . f_a
// (either term skipped when its mesh pointer is null).
__global__ void k_adjoint_gather_f64(const double* __restrict__ x, const double* __restrict__ y,
                                     const double* __restrict__ z, const double* __restrict__ dbar,
                                     double scale_d, const double* __restrict__ ux,
                                     const double* __restrict__ uy, const double* __restrict__ uz,
                                     const double* __restrict__ fx, const double* __restrict__ fy,
                                     const double* __restrict__ fz, double scale_u, double* __restrict__ bx,
                                     double* __restrict__ by, double* __restrict__ bz, long long np, int n) {
    const double dn = (double)n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        const double xp = wrapped(x[p], dn), yp = wrapped(y[p], dn), zp = wrapped(z[p], dn);
        const double flx = floor(xp), fly = floor(yp), flz = floor(zp);
        const int i0 = (int)flx, j0 = (int)fly, k0 = (int)flz;
        const double tx = xp - flx, ty = yp - fly, tz = zp - flz;
        double sx = 0.0, sy = 0.0, sz = 0.0, gx, gy, gz;
        if (dbar) {
            grad_gather(dbar, n + 2, n, i0, j0, k0, tx, ty, tz, gx, gy, gz);
            sx += scale_d * gx;
            sy += scale_d * gy;
            sz += scale_d * gz;
        }
        if (fx) {
            const double u[3] = {ux[p], uy[p], uz[p]};
            const double* f[3] = {fx, fy, fz};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                grad_gather(f[a], n, n, i0, j0, k0, tx, ty, tz, gx, gy, gz);
                sx += scale_u * u[a] * gx;
                sy += scale_u * u[a] * gy;
                sz += scale_u * u[a] * gz;
            }
        }
        bx[p] += sx;
        by[p] += sy;
        bz[p] += sz;
    }
}

__global__ void k_axpy3_f64(double* __restrict__ yx, double* __restrict__ yy, double* __restrict__ yz,
                            const double* __restrict__ xx, const double* __restrict__ xy,
                            const double* __restrict__ xz, double a, long long np) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np;
         p += (long long)gridDim.x * blockDim.x) {
        yx[p] += a * xx[p];
        yy[p] += a * xy[p];
        yz[p] += a * xz[p];
    }
}

}  // namespace

int adjoint_gather_f64(const Plan& p, const double* x, const double* y, const double* z, const double* dbar,
                       double scale_d, const double* u[3], const double* f[3], double scale_u, double* bx,
                       double* by, double* bz, int64_t np) {
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_ADJOINT);
        k_adjoint_gather_f64<<<grid_for(p, np, 256), 256, 0, p.stream>>>(
            x, y, z, dbar, scale_d, u ? u[0] : nullptr, u ? u[1] : nullptr, u ? u[2] : nullptr,
            f ? f[0] : nullptr, f ? f[1] : nullptr, f ? f[2] : nullptr, scale_u, bx, by, bz, np, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int adjoint_mesh_source_f64(const Plan& p, const double* x, const double* y, const double* z, const double* u[3],
                            int64_t np, double* ub[3], double* phibar) {
    const size_t cells = (size_t)p.ng * p.ng * p.ng;
    for (int a = 0; a < 3; ++a) PMB_CUDA_CHECK(cudaMemsetAsync(ub[a], 0, cells * sizeof(double), p.stream));
    {
        Timed t(p, ST_ADJOINT, np > 0 ? 2 : 1);
        if (np > 0)
            k_deposit3_f64<<<grid_for(p, np, 256), 256, 0, p.stream>>>(x, y, z, u[0], u[1], u[2], np, ub[0], ub[1],
                                                                      ub[2], p.ng);
        if (p.grad_order == 4)
            k_neg_divergence_f64<4><<<grid_for(p, (long long)p.ng * p.ng, 1), 256, 0, p.stream>>>(ub[0], ub[1], ub[2],
                                                                                             phibar, p.ng);
        else
            k_neg_divergence_f64<2><<<grid_for(p, (long long)p.ng * p.ng, 1), 256, 0, p.stream>>>(ub[0], ub[1], ub[2],
                                                                                             phibar, p.ng);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int axpy3_f64(const Plan& p, double* y[3], const double* x[3], double a, int64_t np) {
    if (np == 0) return PM_OK;
    k_axpy3_f64<<<grid_for(p, np, 256), 256, 0, p.stream>>>(y[0], y[1], y[2], x[0], x[1], x[2], a, np);
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

}  // namespace pmb
