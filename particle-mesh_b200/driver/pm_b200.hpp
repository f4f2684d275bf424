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
#include <vector>
#include <cstdio>

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

// ---------------------------------------------- cosmological time stepping
// Leapfrog kick-drift-kick in the scale factor a, the integration the
// reference sketches but does not run (src/utils/utils.cpp:141-143: kick with
// function_a(a) Da at the Poisson prefactor 3 Omega_0 / (2a) of
// src/fft/fftw/fft.cpp:55; drift with a^-2 function_a(a) Da at the half
// step).  Force evaluation s = 0..nsteps happens at a_s = a0 + s da with the
// half kicks of neighbouring steps merged; after evaluation s < nsteps the
// particles drift with a_{s+1/2}.  Each entry is one pm_step_* call.
struct CosmoStep {
    double a, c_poisson, c_kick, dt;
};
inline std::vector<CosmoStep> cosmo_schedule(double a0, double da, int nsteps) {
    std::vector<CosmoStep> out;
    for (int s = 0; s <= nsteps; ++s) {
        const double a = a0 + s * da, ah = a0 + (s + 0.5) * da;
        const double w = (s == 0 || s == nsteps) ? 0.5 : 1.0;
        out.push_back({a, 3.0 * Omega_0 / (2.0 * a), w * function_a(a) * da,
                       s < nsteps ? function_a(ah) * da / (ah * ah) : 0.0});
    }
    return out;
}

// Snapshot file (new; the reference writes no output): little-endian,
// a 72-byte header then six float64 arrays of np values
// (x, y, z in cell units, then the momenta or velocities vx, vy, vz).
//   0  char[8] "PMSNAP1"   8 uint32 version (1)   12 uint32 flags (0)
//   16 int64 ng   24 int64 np   32 double a   40 double mass
//   48 double Omega_m   56 double Omega_lambda   64 double Omega_0
struct SnapshotHeader {
    char magic[8] = {'P', 'M', 'S', 'N', 'A', 'P', '1', '\0'};
    uint32_t version = 1, flags = 0;
    int64_t ng = 0, np = 0;
    double a = 0, mass = 0, omega_m = Omega_m, omega_lambda = Omega_lambda, omega_0 = Omega_0;
};
static_assert(sizeof(SnapshotHeader) == 72, "snapshot header layout");

// Writes the snapshot from six host arrays of np doubles.
inline void write_snapshot(const char* path, int ng, double a, double mass, const double* const host[6], size_t np) {
    FILE* f = std::fopen(path, "wb");
    if (!f) throw Error(PM_ERR_ARG, std::string("cannot open ") + path);
    SnapshotHeader h;
    h.ng = ng;
    h.np = static_cast<int64_t>(np);
    h.a = a;
    h.mass = mass;
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1;
    for (int c = 0; c < 6 && ok; ++c) ok = std::fwrite(host[c], sizeof(double), np, f) == np;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw Error(PM_ERR_ARG, std::string("writing ") + path + " failed");
}

}  // namespace pm
