// pm_main: the reference's benchmark loop (src/core/main.cpp) re-hosted on
// one B200 through the C ABI.
//
//   pm_main Ng Nrow [--steps N] [--warmup W] [--dump FILE]
//           [--cosmo STEPS] [--snapshot FILE]
//
// Same inputs as the reference (main.cpp:18-21): Ng mesh cells per side,
// Nrow^3 particles from init_particles (uniform, seeds 0/1/2), zero momenta,
// a = Start_a, mass = Ng^3 / Np.  Same loop shape: 10 warm-up + 20 timed
// iterations (main.cpp:84-86), and rank 0 prints the mean time of the same
// 9 stage buckets (main.cpp:141-143), one per line, in seconds.  The four
// exchange buckets (Alltoallv, reorder, reorder-back, Alltoallv-back) are 0:
// one GPU holds the whole box.  Stage times come from CUDA events on the
// plan's stream.  --dump writes positions then momenta (6 Np doubles) after
// the run, for checking against the reference.  --cosmo then advances the
// particles by STEPS leapfrog steps in the scale factor from Start_a with
// da = Da (pm::cosmo_schedule, FP64 step, the reference's discrete Green's
// function and 2-point gradient), and --snapshot writes the final state in
// the pm::SnapshotHeader format.
#include <cuda_runtime.h>

#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pm_b200.hpp"

#define CUDA_OK(x)                                                                        \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess) {                                                          \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                 \
            return 2;                                                                     \
        }                                                                                 \
    } while (0)

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s Ng Nrow [--steps N] [--warmup W] [--dump FILE] [--cosmo STEPS] "
                             "[--snapshot FILE]\n", argv[0]);
        return 1;
    }
    const int Ng = std::atoi(argv[1]);
    const int Nrow = std::atoi(argv[2]);
    int loop = 20, worm_up = 10;
    const char* dump = nullptr;
    const char* snapshot = nullptr;
    int cosmo = 0;
    for (int i = 3; i + 1 < argc; i += 2) {
        if (!std::strcmp(argv[i], "--steps")) loop = std::atoi(argv[i + 1]);
        else if (!std::strcmp(argv[i], "--warmup")) worm_up = std::atoi(argv[i + 1]);
        else if (!std::strcmp(argv[i], "--dump")) dump = argv[i + 1];
        else if (!std::strcmp(argv[i], "--cosmo")) cosmo = std::atoi(argv[i + 1]);
        else if (!std::strcmp(argv[i], "--snapshot")) snapshot = argv[i + 1];
    }
    const size_t Ng3 = static_cast<size_t>(Ng) * Ng * Ng;
    const size_t Np = static_cast<size_t>(Nrow) * Nrow * Nrow;
    const double mass = static_cast<double>(Ng3) / static_cast<double>(Np);
    const double a = pm::Start_a;

    try {
        pm::Plan plan(Ng);
        // buffers: mesh [Ng][Ng][Ng+2], three force arrays, particles (main.cpp:42-81)
        double *real_buf, *d[3], *pos[3], *mom[3];
        CUDA_OK(cudaMalloc(&real_buf, sizeof(double) * static_cast<size_t>(Ng) * Ng * (Ng + 2)));
        for (auto& q : d) CUDA_OK(cudaMalloc(&q, sizeof(double) * Ng3));
        for (auto& q : pos) CUDA_OK(cudaMalloc(&q, sizeof(double) * Np));
        for (auto& q : mom) CUDA_OK(cudaMalloc(&q, sizeof(double) * Np));
        std::vector<double> hx(Np), hy(Np), hz(Np);
        pm::init_particles(hx.data(), hy.data(), hz.data(), Np, 0, 0, 0, Ng, Ng, Ng, 0);
        CUDA_OK(cudaMemcpy(pos[0], hx.data(), sizeof(double) * Np, cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(pos[1], hy.data(), sizeof(double) * Np, cudaMemcpyHostToDevice));
        CUDA_OK(cudaMemcpy(pos[2], hz.data(), sizeof(double) * Np, cudaMemcpyHostToDevice));
        for (auto& q : mom) CUDA_OK(cudaMemset(q, 0, sizeof(double) * Np));

        pm::FFT fft(plan, real_buf);
        std::array<double, 9> exe_time{};
        std::vector<double> ms(PM_STAGE_COUNT);
        auto stage = [&](const char* name) {
            for (int s = 0; s < PM_STAGE_COUNT; ++s)
                if (!std::strcmp(pm_stage_name(s), name)) return ms[s];
            return 0.0;
        };
        for (int i = 0; i < worm_up + loop; ++i) {
            pm::check(pm_plan_set_timing(plan.get(), i >= worm_up));
            pm::deposit_particles(plan, pos[0], pos[1], pos[2], Np, real_buf, mass);  // CIC
            fft.forward();                                                            // FFT
            fft.apply_green(a);                                                       // Green
            fft.backward();                                                           // IFFT
            pm::centered_derivatives(plan, real_buf, d[0], d[1], d[2]);               // update
            pm::update_particles(plan, pos[0], pos[1], pos[2], d[0], d[1], d[2], mom[0], mom[1], mom[2], a, Np);
        }
        pm::check(pm_plan_read_timing(plan.get(), ms.data(), nullptr, 1));
        plan.check_positions();
        exe_time[0] = stage("mesh_init") + stage("deposit");
        exe_time[3] = stage("fft_z_r2c") + stage("fft_y_fwd") + stage("fft_x_fwd");
        exe_time[4] = stage("green");
        exe_time[5] = stage("fft_x_inv") + stage("fft_y_inv") + stage("fft_z_c2r");
        exe_time[8] = stage("gradient") + stage("interp_kick");
        for (double t : exe_time) std::printf("%.9g\n", loop > 0 ? t / 1e3 / loop : 0.0);

        if (dump) {
            FILE* f = std::fopen(dump, "wb");
            if (!f) {
                std::fprintf(stderr, "cannot open %s\n", dump);
                return 3;
            }
            std::vector<double> h(Np);
            for (double* src : {pos[0], pos[1], pos[2], mom[0], mom[1], mom[2]}) {
                CUDA_OK(cudaMemcpy(h.data(), src, sizeof(double) * Np, cudaMemcpyDeviceToHost));
                std::fwrite(h.data(), sizeof(double), Np, f);
            }
            std::fclose(f);
        }
        if (cosmo > 0) {
            for (const pm::CosmoStep& c : pm::cosmo_schedule(pm::Start_a, pm::Da, cosmo))
                pm::check(pm_step_f64(plan.get(), pos[0], pos[1], pos[2], mom[0], mom[1], mom[2],
                                      static_cast<int64_t>(Np), mass, c.c_poisson, c.c_kick, c.dt));
            plan.check_positions();
        }
        if (snapshot) {
            std::vector<std::vector<double>> h(6, std::vector<double>(Np));
            const double* dev[6] = {pos[0], pos[1], pos[2], mom[0], mom[1], mom[2]};
            const double* host[6];
            for (int c = 0; c < 6; ++c) {
                CUDA_OK(cudaMemcpy(h[c].data(), dev[c], sizeof(double) * Np, cudaMemcpyDeviceToHost));
                host[c] = h[c].data();
            }
            pm::write_snapshot(snapshot, Ng, pm::Start_a + cosmo * pm::Da, mass, host, Np);
        }
        cudaFree(real_buf);
        for (auto q : d) cudaFree(q);
        for (auto q : pos) cudaFree(q);
        for (auto q : mom) cudaFree(q);
    } catch (const pm::Error& e) {
        std::fprintf(stderr, "pm error %d: %s\n", e.code, e.what());
        return 4;
    }
    return 0;
}
