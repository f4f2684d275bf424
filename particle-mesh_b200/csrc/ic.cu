// Zel'dovich initial conditions on the device (FP64).
//
// New code: the reference only draws uniform positions
// (src/utils/utils.cpp:22-36).  Particles sit on an nrow^3 lattice
// q = (i + 1/2) ng/nrow and are displaced by psi, psi_hat_a = i k_a / k^2
// delta_hat, delta_hat = W_hat |k|^(n_s/2) with W white noise, so that
// P(k) ~ k^n_s; psi is scaled to an rms 3D displacement of rms_cells and the
// velocities are vel_factor * psi.
//
// White noise: key = splitmix64(seed); for lattice site i,
//   u1 = ((splitmix64(key ^ 2i) >> 11) + 1) 2^-53,
//   u2 =  (splitmix64(key ^ (2i+1)) >> 11) 2^-53,
//   g  = sqrt(-2 ln u1) cos(2 pi u2)                  (Box-Muller).
// SplitMix64 is the finaliser of Steele, Lea and Flood (OOPSLA 2014).
#include "pm_internal.cuh"

namespace pmb {

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t splitmix64_host(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_white_noise(double* __restrict__ mesh, int n, uint64_t key) {
    const long long total = (long long)n * n * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const uint64_t h1 = splitmix64(key ^ (2ull * (uint64_t)i));
        const uint64_t h2 = splitmix64(key ^ (2ull * (uint64_t)i + 1ull));
        const double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53;
        const double u2 = (double)(h2 >> 11) * 0x1.0p-53;
        const double g = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        const long long k = i % n, r = i / n;
        mesh[r * (n + 2) + k] = g;
        if (k == 0) {  // padding of this row
            mesh[r * (n + 2) + n] = 0.0;
            mesh[r * (n + 2) + n + 1] = 0.0;
        }
    }
}

// psi_hat_a = i k_a W_hat |k|^(n_s/2) / k^2 / n^3 (the 1/n^3 normalises the
// unnormalised C2R that follows); k_a = 0 on its Nyquist plane.
__global__ void k_zeldovich_filter(double2* __restrict__ w_psix, double2* __restrict__ psiy,
                                   double2* __restrict__ psiz, int n, double n_s) {
    const int h = n / 2 + 1;
    const long long total = (long long)n * n * h;
    const double w = 6.283185307179586476925286766559 / n;
    const double inv_n3 = 1.0 / ((double)n * n * n);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int kz = (int)(i % h);
        const long long r = i / h;
        const int ky = (int)(r % n), kx = (int)(r / n);
        const int mx = kx < n / 2 ? kx : kx - n, my = ky < n / 2 ? ky : ky - n;
        const double fx = w * mx, fy = w * my, fz = w * kz;
        const double k2 = fx * fx + fy * fy + fz * fz;
        double2 ox = make_double2(0, 0), oy = ox, oz = ox;
        if (k2 > 0.0) {
            const double2 W = w_psix[i];
            const double s = pow(k2, n_s / 4.0) / k2 * inv_n3;
            const double dr = W.x * s, di = W.y * s;
            const double ax = kx == n / 2 ? 0.0 : fx, ay = ky == n / 2 ? 0.0 : fy, az = kz == n / 2 ? 0.0 : fz;
            ox = make_double2(-ax * di, ax * dr);
            oy = make_double2(-ay * di, ay * dr);
            oz = make_double2(-az * di, az * dr);
        }
        w_psix[i] = ox;
        psiy[i] = oy;
        psiz[i] = oz;
    }
}

__global__ void k_sumsq(const double* __restrict__ a, const double* __restrict__ b,
                        const double* __restrict__ c, int n, double* __restrict__ out) {
    const long long total = (long long)n * n * n;
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long o = (i / n) * (n + 2) + i % n;
        s += a[o] * a[o] + b[o] * b[o] + c[o] * c[o];
    }
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) atomicAdd(out, s);
    }
}

__device__ __forceinline__ double np_mod(double v, double n) {
    double m = fmod(v, n);
    if (m < 0.0) m += n;
    if (m >= n) m -= n;
    return m;
}

__global__ void k_ic_particles(const double* __restrict__ px, const double* __restrict__ py,
                               const double* __restrict__ pz, int nrow, int ng,
                               const double* __restrict__ sumsq, double rms_cells, double vel_factor,
                               double* __restrict__ x, double* __restrict__ y, double* __restrict__ z,
                               double* __restrict__ vx, double* __restrict__ vy, double* __restrict__ vz) {
    const long long total = (long long)nrow * nrow * nrow;
    const double sp = (double)ng / (double)nrow;
    const double rms = sqrt(*sumsq / (double)total) * sp;
    const double s = sp * (rms > 0.0 ? rms_cells / rms : 0.0);
    const double dn = (double)ng;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % nrow), j = (int)((i / nrow) % nrow), a = (int)(i / ((long long)nrow * nrow));
        const long long o = (i / nrow) * (nrow + 2) + k;
        const double dx = px[o] * s, dy = py[o] * s, dz = pz[o] * s;
        x[i] = np_mod((a + 0.5) * sp + dx, dn);
        y[i] = np_mod((j + 0.5) * sp + dy, dn);
        z[i] = np_mod((k + 0.5) * sp + dz, dn);
        vx[i] = vel_factor * dx;
        vy[i] = vel_factor * dy;
        vz[i] = vel_factor * dz;
    }
}

}  // namespace

int ic_zeldovich(const Plan& p, double n_s, double rms_cells, uint64_t seed, double vel_factor, int ng,
                 double* x, double* y, double* z, double* vx, double* vy, double* vz) {
    const int n = p.ng;
    const size_t me = mesh_elems(n);
    double* m[3] = {nullptr, nullptr, nullptr};
    double* sum = nullptr;
    int rc = PM_OK;
    for (int a = 0; a < 3 && rc == PM_OK; ++a)
        if (cudaMalloc(&m[a], me * sizeof(double)) != cudaSuccess) rc = fail(PM_ERR_NOMEM, "ic: mesh allocation failed");
    if (rc == PM_OK && cudaMalloc(&sum, sizeof(double)) != cudaSuccess) rc = fail(PM_ERR_NOMEM, "ic: allocation failed");
    if (rc == PM_OK) {
        const long long cells = (long long)n * n * n;
        const long long modes = (long long)n * n * (n / 2 + 1);
        k_white_noise<<<grid_for(p, cells, 256), 256, 0, p.stream>>>(m[0], n, splitmix64_host(seed));
        rc = fft_r2c<double>(p, m[0]);
        if (rc == PM_OK) {
            k_zeldovich_filter<<<grid_for(p, modes, 256), 256, 0, p.stream>>>(
                reinterpret_cast<double2*>(m[0]), reinterpret_cast<double2*>(m[1]), reinterpret_cast<double2*>(m[2]), n, n_s);
            for (int a = 0; a < 3 && rc == PM_OK; ++a) rc = fft_c2r<double>(p, m[a]);
        }
        if (rc == PM_OK) {
            cudaMemsetAsync(sum, 0, sizeof(double), p.stream);
            k_sumsq<<<grid_for(p, cells, 256), 256, 0, p.stream>>>(m[0], m[1], m[2], n, sum);
            k_ic_particles<<<grid_for(p, cells, 256), 256, 0, p.stream>>>(m[0], m[1], m[2], n, ng, sum, rms_cells,
                                                                         vel_factor, x, y, z, vx, vy, vz);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(p.stream);
            if (e != cudaSuccess) rc = cuda_fail(e, "ic kernels");
        }
    }
    cudaStreamSynchronize(p.stream);
    for (double* a : m)
        if (a) cudaFree(a);
    if (sum) cudaFree(sum);
    return rc;
}

}  // namespace pmb
