// C++ host side of the B200 particle-mesh step, over the C ABI of
// include/pm_b200.h.
//
// The free functions and the FFT class keep the names, argument meaning and
// call order of the reference's CPU interface (include/utils/utils.h:3-10,
// include/fft/fftw/fft.h:10-48) so its stage loop (src/core/main.cpp:90-139)
// ports line for line.  Differences, all forced by one GPU and no MPI:
//   * arrays are device pointers; the plan carries mesh size and stream;
//   * there is no slab / cube bookkeeping (x0, nx_loc, ...): one rank owns
//     the whole periodic box, so the Alltoallv / reorder stages vanish;
//   * every call checks its arguments and throws pm::Error on failure where
//     the reference has no error reporting at all.
#pragma once

#include <cstddef>
#include <cmath>
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>

#include "pm_b200.h"

namespace pm {

// include/utils/utils_inline.h:13-17
constexpr double Omega_0 = 1.0, Omega_m = 0.3, Omega_lambda = 0.7;
constexpr double Omega_k = 1 - Omega_m - Omega_lambda;
constexpr double Da = 0.001, Start_a = 0.9;

// include/utils/utils_inline.h:51-53
inline double function_a(double a) { return 1.0 / std::sqrt(Omega_m / a + Omega_k + Omega_lambda * a * a); }

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != PM_OK) throw Error(rc, pm_last_error());
}

// One periodic ng^3 box (pm_plan_create / pm_plan_destroy).
class Plan {
public:
    Plan(int ng, int precision = PM_FP64, int green = PM_GREEN_DISCRETE, int grad_order = 2,
         void* stream = nullptr)
        : ng_(ng) {
        check(pm_plan_create(ng, precision, green, grad_order, stream, &p_));
    }
    ~Plan() { pm_plan_destroy(p_); }
    Plan(const Plan&) = delete;
    Plan& operator=(const Plan&) = delete;
    pm_plan* get() const { return p_; }
    int ng() const { return ng_; }
    void check_positions() { pm::check(pm_plan_check(p_)); }

private:
    pm_plan* p_ = nullptr;
    int ng_;
};

// init_particles, src/utils/utils.cpp:22-36: uniform positions in the rank's
// cube from three mt19937_64 streams seeded 3r, 3r+1, 3r+2 (host memory).
inline void init_particles(double* posx, double* posy, double* posz, size_t Np_local, int x0, int y0,
                           int z0, int nx_loc, int ny_loc, int nz_loc, int rank) {
    std::mt19937_64 gx(static_cast<uint64_t>(rank) * 3ULL), gy(static_cast<uint64_t>(rank) * 3ULL + 1),
        gz(static_cast<uint64_t>(rank) * 3ULL + 2);
    std::uniform_real_distribution<double> rx(x0, x0 + nx_loc), ry(y0, y0 + ny_loc), rz(z0, z0 + nz_loc);
    for (size_t p = 0; p < Np_local; ++p) {
        posx[p] = rx(gx);
        posy[p] = ry(gy);
        posz[p] = rz(gz);
    }
}

// init_buf + deposit_particles + reduce_private_to_shared + TransposeSlab +
// ReorderSlab (src/utils/utils.cpp:38-113, src/decomp/slab/*): the density
// contrast into buf [ng][ng][ng+2].
inline void deposit_particles(Plan& plan, const double* posx, const double* posy, const double* posz,
                              size_t Np_local, double* buf, double mass) {
    check(pm_deposit_f64(plan.get(), posx, posy, posz, static_cast<int64_t>(Np_local), mass, buf));
}

// class FFT, include/fft/fftw/fft.h:10-48: in-place R2C / C2R of buf and the
// Green's function of src/fft/fftw/fft.cpp:50-57 applied with 1/a.
class FFT {
public:
    FFT(Plan& plan, double* buf) : plan_(plan), buf_(buf) {}
    void forward() { check(pm_fft_r2c_f64(plan_.get(), buf_)); }
    void backward() { check(pm_fft_c2r_f64(plan_.get(), buf_)); }
    void apply_green(const double a) const { check(pm_green_f64(plan_.get(), buf_, 3.0 * Omega_0 / (2.0 * a))); }
    ptrdiff_t local_n0() const { return plan_.ng(); }
    ptrdiff_t local_0_start() const { return 0; }
    ptrdiff_t local_alloc() const {
        return static_cast<ptrdiff_t>(plan_.ng()) * plan_.ng() * (plan_.ng() / 2 + 1);
    }

private:
    Plan& plan_;
    double* buf_;
};

// ReorderSlabBack + TransposeSlabBack + centered_derivatives
// (src/decomp/slab/*_back.cpp, src/utils/utils.cpp:115-137).
inline void centered_derivatives(Plan& plan, const double* in, double* d_dx, double* d_dy, double* d_dz) {
    check(pm_gradient_f64(plan.get(), in, d_dx, d_dy, d_dz));
}

// update_particles, src/utils/utils.cpp:141-170.
inline void update_particles(Plan& plan, const double* posx, const double* posy, const double* posz,
                             const double* d_dx, const double* d_dy, const double* d_dz, double* px,
                             double* py, double* pz, const double a, const size_t Np_local) {
    check(pm_interp_kick_f64(plan.get(), posx, posy, posz, d_dx, d_dy, d_dz, px, py, pz,
                             static_cast<int64_t>(Np_local), function_a(a) * Da));
}

}  // namespace pm
