// Internal declarations shared by the CUDA translation units of the
// particle-mesh step.  Not part of the C ABI (that is include/pm_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/pm_b200.h"

namespace pmb {

// ------------------------------------------------------------ complex types
template <typename T> struct Cx;
template <> struct Cx<float> { using t = float2; };
template <> struct Cx<double> { using t = double2; };

template <typename C> __host__ __device__ __forceinline__ C cmake(decltype(C::x) a, decltype(C::x) b) {
    C c;
    c.x = a;
    c.y = b;
    return c;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmake<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmake<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return cmake<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmake<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return cmake<C>(a.x * s, a.y * s); }

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
// FP32 complex arithmetic on the paired f32x2 pipe of sm_100 (one
// instruction per complex add / sub, two per multiply-by-constant).
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
template <> __device__ __forceinline__ float2 cmul<float2>(float2 a, float2 b) {
    const float2 t = __fmul2_rn(make_float2(a.x, a.x), b);
    return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), t);
}
template <> __device__ __forceinline__ float2 cscale<float2>(float2 a, float s) {
    return __fmul2_rn(a, make_float2(s, s));
}
#endif

// Periodic wrap of a cell index into [0, n) for any n (the FP32 path also
// serves mixed-radix meshes such as 48 or 80 cells); one compare each way in the
// common case.
__host__ __device__ __forceinline__ int wrap_cell(int c, int n) {
    if (c < 0) c += n;
    else if (c >= n) c -= n;
    if (c < 0 || c >= n) c = ((c % n) + n) % n;
    return c;
}

// ------------------------------------------------------------------- errors
enum : int { ERRBIT_RANGE = 1 };

// Thread-local last-error message, set by the C-ABI layer.
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define PMB_CUDA_CHECK(expr)                                            \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::pmb::cuda_fail(_e, #expr);      \
    } while (0)

// ------------------------------------------------------------ stage timers
// Per-kernel CUDA-event timers and launch counters of a plan (the B200 form
// of the reference's per-stage wall-clock buckets, src/utils/utils.cpp:3-20
// and src/core/main.cpp:88-143).  Launch counts are always kept; events are
// recorded only while timing is switched on.
enum Stage : int {
    ST_MESH_INIT, ST_DEPOSIT, ST_FFT_Z_R2C, ST_FFT_Y_FWD, ST_FFT_X_FWD, ST_GREEN, ST_FFT_X_GREEN,
    ST_FFT_X_INV, ST_FFT_Y_INV, ST_FFT_Z_C2R, ST_GRADIENT, ST_INTERP_KICK, ST_DRIFT, ST_KICK_DRIFT,
    ST_INTERP, ST_SPLIT, ST_BIN, ST_SORT, ST_ADJOINT, ST_COUNT
};
const char* stage_name(int st);

struct StageTimers {
    bool on = false;
    struct Rec { int stage; cudaEvent_t a, b; };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    double ms[ST_COUNT] = {};
    long long launches[ST_COUNT] = {};
    cudaEvent_t get();
    ~StageTimers();
};

// Scratch of the tile-binned deposit and the particle sort (tiles.cu):
// bucket counters, exclusive offsets (nb + 1), scatter cursors, scan block
// sums, and the bucket-ordered particle permutation.
struct TileScratch {
    uint32_t *count = nullptr, *off = nullptr, *cursor = nullptr, *bsum = nullptr, *perm = nullptr;
    long long nb = 0;
    int64_t np_cap = 0;
};

// Where the FFT passes of a decomposed mesh find the elements of a line in
// the transpose buffers: element n of the line of plane p at complex offset
// p * ps + (n >> sl) * s1 + (n & mask) * s0 (the element term below 2^31).
struct LineMap {
    long long ps = 0;
    int s1 = 0, s0 = 0, sl = 0, mask = 0;
};
__host__ __device__ __forceinline__ int lm_off(const LineMap& m, int n) { return (n >> m.sl) * m.s1 + (n & m.mask) * m.s0; }

// Where an FFT pass of a decomposed mesh stores its outputs straight into the
// other ranks' buffers (peer device pointers): element n of the line of plane
// p goes to base[n >> sl] + p * ps + (n & mask) * s0 (complex units; base
// already offset to this rank's block in each destination).
constexpr int kMaxPeers = 16;
struct PeerMap {
    void* base[kMaxPeers] = {};
    long long ps = 0;
    int s0 = 0, sl = 0, mask = 0;
};

// ---------------------------------------------------------------- the plan
struct Plan {
    int ng = 0;
    int precision = PM_FP64;
    int green_kind = PM_GREEN_DISCRETE;
    int grad_order = 2;
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    // Tables of length ng in the plan's precision:
    //   tw[k]  = exp(-2 pi i k / ng)              (twiddles, Green cosines)
    //   g1d[k] = 1D part of -(Laplacian symbol): 4 sin^2(pi k / ng) for the
    //            7-point Laplacian, (2 pi m / ng)^2 (m signed) for spectral
    void* tw = nullptr;
    void* g1d = nullptr;
    int* d_err = nullptr;           // device error bits
    void* mesh = nullptr;           // workspace mesh [ng][ng][ng+2]
    void* force[3] = {nullptr, nullptr, nullptr};  // FP64 force arrays
    void* adj[3] = {nullptr, nullptr, nullptr};    // adjoint source arrays (deposited u), plan precision
    void* adjm = nullptr;                          // FP32 adjoint: the second padded mesh (psi)
    void* red = nullptr;                           // reduction partial sums (FP64)
    void* xspec = nullptr;                         // transposed half spectrum [ky][kx][kz] (ng >= 512)
    size_t bytes = 0;
    StageTimers* timers = nullptr;  // owned by the C-ABI plan object
    TileScratch tiles;
    int tk = 0;  // column-tile width of the strided FFT passes (0: default)
    int rv = 0;  // strided-pass radix split: 0 the default, 1 the alternative (autotuned)
    int gather = PM_GATHER_CACHED;  // gather of pm_step_f32 (pm_plan_set_gather)
};

// Brackets one kernel launch with the plan's stage timer.
struct Timed {
    const Plan& p;
    int st;
    cudaEvent_t a = nullptr;
    Timed(const Plan& plan, int stage, int nlaunch = 1) : p(plan), st(stage) {
        if (!p.timers) return;
        p.timers->launches[st] += nlaunch;
        if (p.timers->on) {
            a = p.timers->get();
            cudaEventRecord(a, p.stream);
        }
    }
    ~Timed() {
        if (a) {
            cudaEvent_t b = p.timers->get();
            cudaEventRecord(b, p.stream);
            p.timers->pending.push_back({st, a, b});
        }
    }
};

inline size_t mesh_elems(int ng) { return (size_t)ng * ng * (ng + 2); }

// FFT passes (fft.cu).  Each returns a PM_* status.
// nbox > 1: a batch of nbox meshes of the plan's size, back to back.
template <typename T> int fft_r2c(const Plan& p, T* mesh, int nbox = 1);
template <typename T> int fft_c2r(const Plan& p, T* mesh, int nbox = 1);
template <typename T> int green_apply(const Plan& p, T* mesh, double c_poisson);
template <typename T> int poisson_fused(const Plan& p, T* mesh, double c_poisson, int nbox = 1);
bool fft_size_supported(int ng);
bool tk_variant_supported(int ng, int precision, int tk);
bool radix_variant_supported(int ng, int precision, int rv);
int strided_radix1(int ng, int rv);
int fft_prepare(const Plan& p);  // one-time kernel attributes (large smem)

// Particle and mesh kernels (particles.cu).
int deposit_f64(const Plan& p, const double* x, const double* y, const double* z, int64_t np,
                double mass, double* mesh);
int gradient_f64(const Plan& p, const double* phi, double* fx, double* fy, double* fz);
int interp_kick_f64(const Plan& p, const double* x, const double* y, const double* z,
                    const double* fx, const double* fy, const double* fz, double* px, double* py,
                    double* pz, int64_t np, double c_kick);
int drift_f64(const Plan& p, double* x, double* y, double* z, const double* px, const double* py,
              const double* pz, int64_t np, double dt);
int split_positions(const Plan& p, const double* x, const double* y, const double* z, int64_t np,
                    uint32_t* cell, float* ox, float* oy, float* oz);
int join_positions(const Plan& p, const uint32_t* cell, const float* ox, const float* oy,
                   const float* oz, int64_t np, double* x, double* y, double* z);
// Tile-binned FP32 deposit and spatial sort (tiles.cu); both may grow the
// plan's tile scratch.
int deposit_f32_tiles(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                      int64_t np, float mass, float* mesh);
int sort_f32(Plan& p, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy, float* vz,
             int64_t np);
int deposit_f32_tiles_batch(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                            const long long* pbeg, const long long* pend, int nbox, int64_t np_total,
                            const float* box_mass, float* mesh);
int kick_drift_f32_batch(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz,
                         float* vx, float* vy, float* vz, const long long* pbeg, const long long* pend, int nbox,
                         int64_t np_total, double c_kick, double dt);
int tile_scratch_ensure(Plan& p, int64_t np, int nbox, long long min_nb = 0);
// Fused deposit + z R2C (tiles.cu) and the rest of the fused Poisson solve
// after it (fft.cu): y forward, x forward + Green + x inverse, y inverse, z C2R.
bool zcol_supported(int ng);
int deposit_zr2c_prepare(const Plan& p);
int deposit_zr2c_f32(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz, int64_t np,
                     float mass, float* mesh, int zcb = 0);
// Gather + kick + drift in the bin order of the last deposit_zr2c_f32 with
// z-chunk bits zcb (chunks of 64 cells, power-of-two ng >= 256), the
// potential staged per block in shared memory (particles.cu).
bool tiled_gather_supported(int ng);
int tiled_gather_zcb(int ng);
int tiled_gather_prepare();
int kick_drift_tiles_f32(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                         float* vy, float* vz, int64_t np, double c_kick, double dt);
int poisson_after_z_f32(const Plan& p, float* mesh, double c_poisson, int nbox = 1);
int deposit_zr2c_f32_batch(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                           const long long* pbeg, const long long* pend, int nbox, int64_t np_total,
                           const float* box_mass, float* mesh);
void tile_scratch_release(Plan& p);
int interp_f32(const Plan& p, const float* phi, const uint32_t* cell, const float* ox,
               const float* oy, const float* oz, int64_t np, float* fx, float* fy, float* fz);
int kick_drift_f32(const Plan& p, const float* phi, uint32_t* cell, float* ox, float* oy, float* oz,
                   float* vx, float* vy, float* vz, int64_t np, double c_kick, double dt);

// x-slab decomposition (tiles.cu, fft.cu, particles.cu, slab.cu).
int slab_deposit_zr2c_f32(Plan& p, int x0, int nx, const uint32_t* cell, const float* ox, const float* oy,
                          const float* oz, int64_t np, float mass, float* mesh);
int slab_rank_sort(Plan& p, int nranks, int nx, const uint32_t* cell, int64_t np, int64_t* counts);
// x-slab FFT passes that read / write the transpose buffers directly (rows
// [ky][x][kz] after the y forward; blocks [rank][kyl][x][kz] around x + Green)
int slab_fft_forward_y_f32(const Plan& p, const float* own, float* send, int nx);
int slab_fft_xgreen_f32(const Plan& p, const float* recv, float* send, double c_poisson, int nx, int ky0);
int slab_fft_backward_f32(const Plan& p, const float* recv, float* own, int nx);
// the same two passes storing into the other ranks' buffers (PeerMap)
int slab_fft_forward_peers_f32(const Plan& p, const float* own, const PeerMap& po, int nx);
int slab_fft_xgreen_peers_f32(const Plan& p, const float* recv, const PeerMap& po, double c_poisson, int nx,
                              int ky0);
int slab_kick_drift_f32(const Plan& p, int x0, int nx, const float* phi, uint32_t* cell, float* ox, float* oy,
                        float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick, double dt);
int plan_create_internal(int ng, int precision, int green_kind, int grad_order, void* stream, pm_plan** out);
// pencil decomposition (tiles.cu, fft.cu, particles.cu, slab.cu)
int pencil_rank_sort(Plan& p, int px, int py, int nx, int ny, const uint32_t* cell, int64_t np, int64_t* counts);
int pencil_copy3(const Plan& p, const float2* src, long long sa, long long sb, float2* dst, long long da, long long db,
                 int A, int B, int C, float bg = 0.0f);
// y lines read / written through line maps; x + Green (kz = kz0 + column,
// ky = ky0 + plane) from `in` to `out` through one map
int pencil_lines_f32(const Plan& p, const float* in, float* out, LineMap mi, LineMap mo, int planes, int ncols,
                     int dir, int stage);
int pencil_xgreen_f32(const Plan& p, const float* in, float* out, LineMap m, int planes, int ncols, double c_poisson,
                      int ky0, int kz0);
int pencil_z_f32(const Plan& p, float* rows, long long nrows, bool forward);
// the same passes storing into the other ranks' buffers
int pencil_lines_peers_f32(const Plan& p, const float* in, LineMap mi, const PeerMap& po, int planes, int ncols,
                           int dir, int stage);
int pencil_xgreen_peers_f32(const Plan& p, const float* in, LineMap m, const PeerMap& po, int planes, int ncols,
                            double c_poisson, int ky0, int kz0);
int pencil_deposit_f32(const Plan& p, int x0, int y0, int nx, int ny, const uint32_t* cell, const float* ox,
                       const float* oy, const float* oz, int64_t np, float mass, float* buf);
int pencil_kick_drift_f32(const Plan& p, int x0, int y0, int nx, int ny, const float* buf, uint32_t* cell, float* ox,
                          float* oy, float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick,
                          double dt);

// Adjoint kernels (adjoint.cu).
int adjoint_gather_f64(const Plan& p, const double* x, const double* y, const double* z, const double* dbar,
                       double scale_d, const double* u[3], const double* f[3], double scale_u, double* bx,
                       double* by, double* bz, int64_t np);
int adjoint_mesh_source_f64(const Plan& p, const double* x, const double* y, const double* z, const double* u[3],
                            int64_t np, double* ub[3], double* phibar);
int axpy3_f64(const Plan& p, double* y[3], const double* x[3], double a, int64_t np);
int adjoint_gather_f32(const Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                       int64_t np, const float* dbar, double scale_d, const float* phi, const float* u[3],
                       double scale_u, float* xbar[3]);
int adjoint_mesh_source_f32(const Plan& p, const uint32_t* cell, const float* ox, const float* oy,
                            const float* oz, const float* u[3], int64_t np, float* ub[3], float* phibar);
int axpy3_f32(const Plan& p, float* y[3], const float* x[3], double a, int64_t np);
template <typename T>
int reduce_conserved(Plan& p, const T* mesh, const T* vx, const T* vy, const T* vz, int64_t np, double mass,
                     double* out);

// Zel'dovich initial conditions (ic.cu); p is an FP64 plan of size nrow.
int ic_zeldovich(const Plan& p, double n_s, double rms_cells, uint64_t seed, double vel_factor, int ng,
                 double* x, double* y, double* z, double* vx, double* vy, double* vz);

// Grid size for a grid-stride loop over n items: whole waves of the SM count.
inline unsigned grid_for(const Plan& p, long long n, int threads, int blocks_per_sm = 8) {
    long long need = (n + threads - 1) / threads;
    long long cap = (long long)p.num_sms * blocks_per_sm;
    if (need < 1) need = 1;
    return (unsigned)(need < cap ? need : cap);
}

}  // namespace pmb

struct pm_plan {
    pmb::Plan p;
};
