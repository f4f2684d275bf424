// C ABI of the particle-mesh step (declared in include/pm_b200.h): argument
// checks, plan lifetime, workspace, and the per-stage / whole-step entry
// points.  All checks happen on the host before anything is enqueued; a
// device-side bad position is recorded in the plan's error word and
// reported by pm_plan_check.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pm_internal.cuh"

namespace pmb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* what) {
    return fail(PM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static const char* kStageNames[ST_COUNT] = {
    "mesh_init", "deposit", "fft_z_r2c", "fft_y_fwd", "fft_x_fwd", "green", "fft_x_green",
    "fft_x_inv", "fft_y_inv", "fft_z_c2r", "gradient", "interp_kick", "drift", "kick_drift",
    "interp", "split", "bin", "sort", "adjoint"};

const char* stage_name(int st) { return st >= 0 && st < ST_COUNT ? kStageNames[st] : ""; }

cudaEvent_t StageTimers::get() {
    if (pool.empty()) {
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
}

StageTimers::~StageTimers() {
    for (auto& r : pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : pool) cudaEventDestroy(e);
}

namespace {

template <typename T> int upload_tables(Plan& p) {
    using C = typename Cx<T>::t;
    const int n = p.ng;
    std::vector<C> tw(n);
    std::vector<T> g1d(n);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; ++k) {
        const long double a = -2.0L * pi * (long double)k / (long double)n;
        tw[k] = cmake<C>((T)cosl(a), (T)sinl(a));
        if (p.green_kind == PM_GREEN_DISCRETE) {
            const long double s = sinl(pi * (long double)k / (long double)n);
            g1d[k] = (T)(4.0L * s * s);
        } else {
            const long double m = k <= n / 2 ? (long double)k : (long double)(k - n);
            const long double w = 2.0L * pi * m / (long double)n;
            g1d[k] = (T)(w * w);
        }
    }
    PMB_CUDA_CHECK(cudaMalloc(&p.tw, n * sizeof(C)));
    PMB_CUDA_CHECK(cudaMalloc(&p.g1d, n * sizeof(T)));
    PMB_CUDA_CHECK(cudaMemcpy(p.tw, tw.data(), n * sizeof(C), cudaMemcpyHostToDevice));
    PMB_CUDA_CHECK(cudaMemcpy(p.g1d, g1d.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    p.bytes += n * (sizeof(C) + sizeof(T));
    return PM_OK;
}

void release(Plan& p) {
    if (p.tw) cudaFree(p.tw);
    if (p.g1d) cudaFree(p.g1d);
    if (p.d_err) cudaFree(p.d_err);
    if (p.mesh) cudaFree(p.mesh);
    for (void*& f : p.force)
        if (f) cudaFree(f), f = nullptr;
    for (void*& f : p.adj)
        if (f) cudaFree(f), f = nullptr;
    if (p.adjm) cudaFree(p.adjm);
    if (p.red) cudaFree(p.red);
    if (p.xspec) cudaFree(p.xspec);
    p.tw = p.g1d = p.mesh = p.adjm = p.red = p.xspec = nullptr;
    p.d_err = nullptr;
    delete p.timers;
    p.timers = nullptr;
    tile_scratch_release(p);
}

// FP32 plans of a power-of-two mesh >= 512 get the transposed half spectrum
// that lets the x + Green pass write its lines at element stride H (the
// Poisson solve runs in place without it, e.g. when this allocation fails).
void ensure_xspec(Plan& p) {
    if (p.xspec || p.precision != PM_FP32 || p.ng < 512 || (p.ng & (p.ng - 1)) != 0) return;
    const size_t b = (size_t)p.ng * p.ng * (p.ng / 2 + 1) * 2 * sizeof(float);
    if (cudaMalloc(&p.xspec, b) != cudaSuccess) {
        cudaGetLastError();
        p.xspec = nullptr;
        return;
    }
    p.bytes += b;
}

int ensure_workspace(Plan& p, bool forces, bool adjoint = false) {
    const size_t esz = p.precision == PM_FP64 ? sizeof(double) : sizeof(float);
    ensure_xspec(p);
    if (!p.mesh) {
        if (cudaMalloc(&p.mesh, mesh_elems(p.ng) * esz) != cudaSuccess) {
            cudaGetLastError();
            p.mesh = nullptr;
            return fail(PM_ERR_NOMEM, "workspace mesh allocation failed");
        }
        p.bytes += mesh_elems(p.ng) * esz;
    }
    if (forces && !p.force[0]) {
        const size_t b = (size_t)p.ng * p.ng * p.ng * sizeof(double);
        for (void*& f : p.force) {
            if (cudaMalloc(&f, b) != cudaSuccess) {
                cudaGetLastError();
                f = nullptr;
                return fail(PM_ERR_NOMEM, "workspace force allocation failed");
            }
            p.bytes += b;
        }
    }
    if (adjoint && !p.adj[0]) {
        const size_t b = (size_t)p.ng * p.ng * p.ng * esz;
        for (void*& f : p.adj) {
            if (cudaMalloc(&f, b) != cudaSuccess) {
                cudaGetLastError();
                f = nullptr;
                return fail(PM_ERR_NOMEM, "adjoint workspace allocation failed");
            }
            p.bytes += b;
        }
    }
    // FP32 keeps phi for the direct term, so the adjoint potential needs a
    // padded mesh of its own (FP64 reuses the plan mesh after the gradient)
    if (adjoint && p.precision == PM_FP32 && !p.adjm) {
        if (cudaMalloc(&p.adjm, mesh_elems(p.ng) * esz) != cudaSuccess) {
            cudaGetLastError();
            p.adjm = nullptr;
            return fail(PM_ERR_NOMEM, "adjoint workspace allocation failed");
        }
        p.bytes += mesh_elems(p.ng) * esz;
    }
    return PM_OK;
}

int check_plan(const pm_plan* plan, int precision) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    if (plan->p.precision != precision)
        return fail(PM_ERR_STATE, precision == PM_FP64 ? "entry point needs a PM_FP64 plan"
                                                       : "entry point needs a PM_FP32 plan");
    return PM_OK;
}

int check_np(int64_t np, std::initializer_list<const void*> ptrs) {
    if (np < 0) return fail(PM_ERR_ARG, "negative particle count");
    if (np > 0)
        for (const void* q : ptrs)
            if (!q) return fail(PM_ERR_ARG, "NULL particle array");
    return PM_OK;
}

int set_device(const Plan& p) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail(PM_ERR_CUDA, "cudaGetDevice failed");
    if (cur != p.device) PMB_CUDA_CHECK(cudaSetDevice(p.device));
    return PM_OK;
}

}  // namespace
}  // namespace pmb

using namespace pmb;

#define PM_TRY(expr)                 \
    do {                             \
        int _rc = (expr);            \
        if (_rc != PM_OK) return _rc; \
    } while (0)

extern "C" {

const char* pm_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

static int plan_create(int ng, int precision, int green_kind, int grad_order, void* stream, pm_plan** out) {
    if (!out) return fail(PM_ERR_ARG, "output pointer is NULL");
    *out = nullptr;
    if (!fft_size_supported(ng))
        return fail(PM_ERR_SIZE,
                    "ng must be a power of two in [8, 1024] or one of the mixed-radix sizes 24, 40, 48, 80, 96, 120, "
                    "160, 192, 240, 320, 384, 480, 640, 768, 960");
    if (precision != PM_FP64 && precision != PM_FP32) return fail(PM_ERR_ARG, "unknown precision");
    if (green_kind != PM_GREEN_DISCRETE && green_kind != PM_GREEN_SPECTRAL) return fail(PM_ERR_ARG, "unknown green_kind");
    if (grad_order != 2 && grad_order != 4) return fail(PM_ERR_ARG, "grad_order must be 2 or 4");
    pm_plan* plan = new (std::nothrow) pm_plan();
    if (!plan) return fail(PM_ERR_NOMEM, "host allocation failed");
    Plan& p = plan->p;
    p.ng = ng;
    p.precision = precision;
    p.green_kind = green_kind;
    p.grad_order = grad_order;
    p.stream = static_cast<cudaStream_t>(stream);
    int rc = PM_OK;
    if (cudaGetDevice(&p.device) != cudaSuccess) rc = fail(PM_ERR_CUDA, "no CUDA device");
    if (rc == PM_OK && cudaDeviceGetAttribute(&p.num_sms, cudaDevAttrMultiProcessorCount, p.device) != cudaSuccess)
        rc = fail(PM_ERR_CUDA, "cudaDeviceGetAttribute failed");
    if (rc == PM_OK) rc = precision == PM_FP64 ? upload_tables<double>(p) : upload_tables<float>(p);
    if (rc == PM_OK) {
        if (cudaMalloc(&p.d_err, sizeof(int)) != cudaSuccess || cudaMemset(p.d_err, 0, sizeof(int)) != cudaSuccess)
            rc = fail(PM_ERR_NOMEM, "error word allocation failed");
    }
    if (rc == PM_OK) rc = fft_prepare(p);
    if (rc == PM_OK && precision == PM_FP32) rc = deposit_zr2c_prepare(p);
    if (rc == PM_OK && precision == PM_FP32 && tiled_gather_supported(ng)) rc = tiled_gather_prepare();
    if (rc == PM_OK) {
        p.timers = new (std::nothrow) StageTimers();
        if (!p.timers) rc = fail(PM_ERR_NOMEM, "host allocation failed");
    }
    if (rc != PM_OK) {
        cudaGetLastError();
        release(p);
        delete plan;
        return rc;
    }
    *out = plan;
    return PM_OK;
}

namespace pmb {
int plan_create_internal(int ng, int precision, int green_kind, int grad_order, void* stream, pm_plan** out) {
    return plan_create(ng, precision, green_kind, grad_order, stream, out);
}
}  // namespace pmb

extern "C" {

int pm_plan_create(int ng, int precision, int green_kind, int grad_order, void* stream, pm_plan** out) {
    return plan_create(ng, precision, green_kind, grad_order, stream, out);
}

int pm_plan_destroy(pm_plan* plan) {
    if (!plan) return PM_OK;
    set_device(plan->p);
    cudaStreamSynchronize(plan->p.stream);
    release(plan->p);
    delete plan;
    return PM_OK;
}

int pm_plan_device_bytes(const pm_plan* plan, size_t* bytes) {
    if (!plan || !bytes) return fail(PM_ERR_ARG, "NULL argument");
    *bytes = plan->p.bytes;
    return PM_OK;
}

int pm_plan_check(pm_plan* plan) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    PM_TRY(set_device(plan->p));
    int h = 0;
    PMB_CUDA_CHECK(cudaStreamSynchronize(plan->p.stream));
    PMB_CUDA_CHECK(cudaMemcpy(&h, plan->p.d_err, sizeof(int), cudaMemcpyDeviceToHost));
    PMB_CUDA_CHECK(cudaMemset(plan->p.d_err, 0, sizeof(int)));
    if (h & ERRBIT_RANGE) return fail(PM_ERR_RANGE, "a particle position was NaN or outside [0, ng); it was wrapped");
    return PM_OK;
}

int pm_plan_set_fft_shape(pm_plan* plan, int tile_cols, int radix1) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    Plan& p = plan->p;
    if (!tk_variant_supported(p.ng, p.precision, tile_cols))
        return fail(PM_ERR_ARG, "tile_cols must be 0, or 8 / 16 / 32 on an FP32 plan with ng <= 128");
    int rv = -1;
    if (radix1 == 0 || radix1 == strided_radix1(p.ng, 0)) rv = 0;
    else if (radix_variant_supported(p.ng, p.precision, 1) && radix1 == strided_radix1(p.ng, 1)) rv = 1;
    if (rv < 0) return fail(PM_ERR_ARG, "radix1 is not a split of this plan's strided passes");
    p.tk = tile_cols;
    p.rv = rv;
    return PM_OK;
}

int pm_plan_set_gather(pm_plan* plan, int mode) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    if (mode != PM_GATHER_CACHED && mode != PM_GATHER_TILED) return fail(PM_ERR_ARG, "unknown gather mode");
    if (mode == PM_GATHER_TILED && (plan->p.precision != PM_FP32 || !tiled_gather_supported(plan->p.ng)))
        return fail(PM_ERR_SIZE, "the tiled gather needs an FP32 plan of a power-of-two ng in [256, 1024]");
    plan->p.gather = mode;
    return PM_OK;
}

int pm_plan_set_timing(pm_plan* plan, int on) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    plan->p.timers->on = on != 0;
    return PM_OK;
}

int pm_plan_read_timing(pm_plan* plan, double* ms, int64_t* launches, int reset) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    PM_TRY(set_device(plan->p));
    StageTimers& t = *plan->p.timers;
    if (!t.pending.empty()) PMB_CUDA_CHECK(cudaStreamSynchronize(plan->p.stream));
    for (auto& r : t.pending) {
        float e = 0.f;
        if (cudaEventElapsedTime(&e, r.a, r.b) == cudaSuccess) t.ms[r.stage] += e;
        t.pool.push_back(r.a);
        t.pool.push_back(r.b);
    }
    t.pending.clear();
    for (int i = 0; i < ST_COUNT; ++i) {
        if (ms) ms[i] = t.ms[i];
        if (launches) launches[i] = t.launches[i];
        if (reset) {
            t.ms[i] = 0.0;
            t.launches[i] = 0;
        }
    }
    return PM_OK;
}

const char* pm_stage_name(int stage) { return stage_name(stage); }

int pm_plan_mesh(pm_plan* plan, void** mesh) {
    if (!plan || !mesh) return fail(PM_ERR_ARG, "NULL argument");
    PM_TRY(set_device(plan->p));
    PM_TRY(ensure_workspace(plan->p, false));
    *mesh = plan->p.mesh;
    return PM_OK;
}

// ------------------------------------------------------------------ FP64

int pm_deposit_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                   double mass, double* mesh) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z}));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return deposit_f64(plan->p, x, y, z, np, mass, mesh);
}

int pm_fft_r2c_f64(pm_plan* plan, double* mesh) {
    PM_TRY(check_plan(plan, PM_FP64));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return fft_r2c<double>(plan->p, mesh);
}

int pm_green_f64(pm_plan* plan, double* mesh, double c_poisson) {
    PM_TRY(check_plan(plan, PM_FP64));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return green_apply<double>(plan->p, mesh, c_poisson);
}

int pm_fft_c2r_f64(pm_plan* plan, double* mesh) {
    PM_TRY(check_plan(plan, PM_FP64));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return fft_c2r<double>(plan->p, mesh);
}

int pm_poisson_f64(pm_plan* plan, double* mesh, double c_poisson) {
    PM_TRY(check_plan(plan, PM_FP64));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return poisson_fused<double>(plan->p, mesh, c_poisson);
}

int pm_gradient_f64(pm_plan* plan, const double* phi, double* fx, double* fy, double* fz) {
    PM_TRY(check_plan(plan, PM_FP64));
    if (!phi || !fx || !fy || !fz) return fail(PM_ERR_ARG, "NULL mesh");
    PM_TRY(set_device(plan->p));
    return gradient_f64(plan->p, phi, fx, fy, fz);
}

int pm_interp_kick_f64(pm_plan* plan, const double* x, const double* y, const double* z,
                       const double* fx, const double* fy, const double* fz, double* px, double* py,
                       double* pz, int64_t np, double c_kick) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, px, py, pz}));
    if (!fx || !fy || !fz) return fail(PM_ERR_ARG, "NULL force mesh");
    PM_TRY(set_device(plan->p));
    return interp_kick_f64(plan->p, x, y, z, fx, fy, fz, px, py, pz, np, c_kick);
}

int pm_drift_f64(pm_plan* plan, double* x, double* y, double* z, const double* px,
                 const double* py, const double* pz, int64_t np, double dt) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, px, py, pz}));
    PM_TRY(set_device(plan->p));
    return drift_f64(plan->p, x, y, z, px, py, pz, np, dt);
}

int pm_step_f64(pm_plan* plan, double* x, double* y, double* z, double* px, double* py,
                double* pz, int64_t np, double mass, double c_poisson, double c_kick, double dt) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, px, py, pz}));
    PM_TRY(set_device(plan->p));
    Plan& p = plan->p;
    PM_TRY(ensure_workspace(p, true));
    double* m = static_cast<double*>(p.mesh);
    double* f[3] = {static_cast<double*>(p.force[0]), static_cast<double*>(p.force[1]),
                    static_cast<double*>(p.force[2])};
    PM_TRY(deposit_f64(p, x, y, z, np, mass, m));
    PM_TRY(fft_r2c<double>(p, m));
    PM_TRY(green_apply<double>(p, m, c_poisson));
    PM_TRY(fft_c2r<double>(p, m));
    PM_TRY(gradient_f64(p, m, f[0], f[1], f[2]));
    PM_TRY(interp_kick_f64(p, x, y, z, f[0], f[1], f[2], px, py, pz, np, c_kick));
    if (dt != 0.0) PM_TRY(drift_f64(p, x, y, z, px, py, pz, np, dt));
    return PM_OK;
}

// ------------------------------------------------------- FP64 adjoints

int pm_adjoint_deposit_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                           double mass, const double* dbar, double* xbar, double* ybar, double* zbar) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, xbar, ybar, zbar}));
    if (!dbar) return fail(PM_ERR_ARG, "dbar is NULL");
    PM_TRY(set_device(plan->p));
    return adjoint_gather_f64(plan->p, x, y, z, dbar, mass, nullptr, nullptr, 0.0, xbar, ybar, zbar, np);
}

// Recomputes the force meshes at x (fused Poisson solve), builds the mesh
// source -sum_a G_a D_a(u) in the same padded mesh once phi is no longer
// needed, solves it with the same (symmetric) Green's operator, and adds the
// direct and mesh terms in one gather.
static int adjoint_force(Plan& p, const double* x, const double* y, const double* z, int64_t np, double mass,
                         double c_poisson, const double* ux, const double* uy, const double* uz, double scale,
                         double* xbar, double* ybar, double* zbar) {
    PM_TRY(ensure_workspace(p, true, true));
    double* m = static_cast<double*>(p.mesh);
    double* f[3] = {static_cast<double*>(p.force[0]), static_cast<double*>(p.force[1]),
                    static_cast<double*>(p.force[2])};
    double* ub[3] = {static_cast<double*>(p.adj[0]), static_cast<double*>(p.adj[1]),
                     static_cast<double*>(p.adj[2])};
    const double* fc[3] = {f[0], f[1], f[2]};
    const double* u[3] = {ux, uy, uz};
    PM_TRY(deposit_f64(p, x, y, z, np, mass, m));
    PM_TRY(poisson_fused<double>(p, m, c_poisson));
    PM_TRY(gradient_f64(p, m, f[0], f[1], f[2]));
    PM_TRY(adjoint_mesh_source_f64(p, x, y, z, u, np, ub, m));
    PM_TRY(poisson_fused<double>(p, m, c_poisson));
    return adjoint_gather_f64(p, x, y, z, m, scale * mass, u, fc, scale, xbar, ybar, zbar, np);
}

int pm_adjoint_force_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                         double mass, double c_poisson, const double* ux, const double* uy, const double* uz,
                         double scale, double* xbar, double* ybar, double* zbar) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, ux, uy, uz, xbar, ybar, zbar}));
    PM_TRY(set_device(plan->p));
    return adjoint_force(plan->p, x, y, z, np, mass, c_poisson, ux, uy, uz, scale, xbar, ybar, zbar);
}

int pm_step_adjoint_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                        double mass, double c_poisson, double c_kick, double dt, double* xbar, double* ybar,
                        double* zbar, double* vxbar, double* vybar, double* vzbar) {
    PM_TRY(check_plan(plan, PM_FP64));
    PM_TRY(check_np(np, {x, y, z, xbar, ybar, zbar, vxbar, vybar, vzbar}));
    PM_TRY(set_device(plan->p));
    Plan& p = plan->p;
    double* vb[3] = {vxbar, vybar, vzbar};
    const double* xb[3] = {xbar, ybar, zbar};
    if (dt != 0.0) PM_TRY(axpy3_f64(p, vb, xb, dt, np));  // x' = x + dt v'  =>  vbar' += dt xbar
    if (c_kick == 0.0) return PM_OK;
    return adjoint_force(p, x, y, z, np, mass, c_poisson, vxbar, vybar, vzbar, c_kick, xbar, ybar, zbar);
}

// ------------------------------------------------------------------ FP32

int pm_split_positions(pm_plan* plan, const double* x, const double* y, const double* z,
                       int64_t np, uint32_t* cell, float* ox, float* oy, float* oz) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    PM_TRY(check_np(np, {x, y, z, cell, ox, oy, oz}));
    PM_TRY(set_device(plan->p));
    return split_positions(plan->p, x, y, z, np, cell, ox, oy, oz);
}

int pm_join_positions(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                      const float* oz, int64_t np, double* x, double* y, double* z) {
    if (!plan) return fail(PM_ERR_ARG, "plan is NULL");
    PM_TRY(check_np(np, {x, y, z, cell, ox, oy, oz}));
    PM_TRY(set_device(plan->p));
    return join_positions(plan->p, cell, ox, oy, oz, np, x, y, z);
}

int pm_deposit_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                   const float* oz, int64_t np, float mass, float* mesh) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz}));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return deposit_f32_tiles(plan->p, cell, ox, oy, oz, np, mass, mesh);
}

int pm_sort_f32(pm_plan* plan, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                float* vz, int64_t np) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, vx, vy, vz}));
    PM_TRY(set_device(plan->p));
    return sort_f32(plan->p, cell, ox, oy, oz, vx, vy, vz, np);
}

int pm_fft_r2c_f32(pm_plan* plan, float* mesh) {
    PM_TRY(check_plan(plan, PM_FP32));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return fft_r2c<float>(plan->p, mesh);
}

int pm_green_f32(pm_plan* plan, float* mesh, double c_poisson) {
    PM_TRY(check_plan(plan, PM_FP32));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return green_apply<float>(plan->p, mesh, c_poisson);
}

int pm_fft_c2r_f32(pm_plan* plan, float* mesh) {
    PM_TRY(check_plan(plan, PM_FP32));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    return fft_c2r<float>(plan->p, mesh);
}

int pm_poisson_f32(pm_plan* plan, float* mesh, double c_poisson) {
    PM_TRY(check_plan(plan, PM_FP32));
    if (!mesh) return fail(PM_ERR_ARG, "mesh is NULL");
    PM_TRY(set_device(plan->p));
    ensure_xspec(plan->p);
    return poisson_fused<float>(plan->p, mesh, c_poisson);
}

int pm_interp_f32(pm_plan* plan, const float* phi, const uint32_t* cell, const float* ox,
                  const float* oy, const float* oz, int64_t np, float* fx, float* fy, float* fz) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, fx, fy, fz}));
    if (!phi) return fail(PM_ERR_ARG, "phi is NULL");
    PM_TRY(set_device(plan->p));
    return interp_f32(plan->p, phi, cell, ox, oy, oz, np, fx, fy, fz);
}

int pm_kick_drift_f32(pm_plan* plan, const float* phi, uint32_t* cell, float* ox, float* oy,
                      float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick,
                      double dt) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, vx, vy, vz}));
    if (!phi) return fail(PM_ERR_ARG, "phi is NULL");
    PM_TRY(set_device(plan->p));
    return kick_drift_f32(plan->p, phi, cell, ox, oy, oz, vx, vy, vz, np, c_kick, dt);
}

// The potential of the particles in the plan's workspace mesh: binning, the
// deposit fused with the z FFT pass (zcb: z-chunk bits of the bins), the
// remaining passes.  Shared by pm_potential_f32 and pm_step_f32.
static int potential_f32(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                         int64_t np, float mass, double c_poisson, int zcb) {
    PM_TRY(ensure_workspace(p, false));
    float* m = static_cast<float*>(p.mesh);
    if (zcol_supported(p.ng)) {  // deposit fused with the z FFT pass
        PM_TRY(deposit_zr2c_f32(p, cell, ox, oy, oz, np, mass, m, zcb));
        return poisson_after_z_f32(p, m, c_poisson);
    }
    PM_TRY(deposit_f32_tiles(p, cell, ox, oy, oz, np, mass, m));
    return poisson_fused<float>(p, m, c_poisson);
}

int pm_potential_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                     int64_t np, float mass, double c_poisson) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz}));
    PM_TRY(set_device(plan->p));
    return potential_f32(plan->p, cell, ox, oy, oz, np, mass, c_poisson, 0);
}

int pm_step_f32(pm_plan* plan, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                float* vy, float* vz, int64_t np, float mass, double c_poisson, double c_kick,
                double dt) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, vx, vy, vz}));
    PM_TRY(set_device(plan->p));
    Plan& p = plan->p;
    float* m = nullptr;
    if (p.gather == PM_GATHER_TILED && tiled_gather_supported(p.ng)) {
        // binned by (column tile, class, z chunk): the deposit fused with the
        // z FFT pass, and the gather from potential tiles staged in shared
        // memory in the same bin order
        PM_TRY(potential_f32(p, cell, ox, oy, oz, np, mass, c_poisson, tiled_gather_zcb(p.ng)));
        m = static_cast<float*>(p.mesh);
        return kick_drift_tiles_f32(p, m, cell, ox, oy, oz, vx, vy, vz, np, c_kick, dt);
    }
    PM_TRY(potential_f32(p, cell, ox, oy, oz, np, mass, c_poisson, 0));
    m = static_cast<float*>(p.mesh);
    return kick_drift_f32(p, m, cell, ox, oy, oz, vx, vy, vz, np, c_kick, dt);
}

// ------------------------------------------------------- FP32 adjoints

int pm_adjoint_deposit_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                           const float* oz, int64_t np, float mass, const float* dbar, float* xbar,
                           float* ybar, float* zbar) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, xbar, ybar, zbar}));
    if (!dbar) return fail(PM_ERR_ARG, "dbar is NULL");
    PM_TRY(set_device(plan->p));
    float* xb[3] = {xbar, ybar, zbar};
    return adjoint_gather_f32(plan->p, cell, ox, oy, oz, np, dbar, mass, nullptr, nullptr, 0.0, xb);
}

// phi at the split positions (the step's own deposit + Poisson path), the
// mesh source -sum_a G_a D_a(u) solved with the same symmetric Green's
// operator into the second mesh, then one gather for both terms.
static int adjoint_force_f32(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                             int64_t np, float mass, double c_poisson, const float* u[3], double scale,
                             float* xbar[3]) {
    PM_TRY(ensure_workspace(p, false, true));
    float* m = static_cast<float*>(p.mesh);
    float* psi = static_cast<float*>(p.adjm);
    float* ub[3] = {static_cast<float*>(p.adj[0]), static_cast<float*>(p.adj[1]), static_cast<float*>(p.adj[2])};
    if (zcol_supported(p.ng)) {
        PM_TRY(deposit_zr2c_f32(p, cell, ox, oy, oz, np, mass, m));
        PM_TRY(poisson_after_z_f32(p, m, c_poisson));
    } else {
        PM_TRY(deposit_f32_tiles(p, cell, ox, oy, oz, np, mass, m));
        PM_TRY(poisson_fused<float>(p, m, c_poisson));
    }
    PM_TRY(adjoint_mesh_source_f32(p, cell, ox, oy, oz, u, np, ub, psi));
    PM_TRY(poisson_fused<float>(p, psi, c_poisson));
    return adjoint_gather_f32(p, cell, ox, oy, oz, np, psi, scale * mass, m, u, scale, xbar);
}

int pm_adjoint_force_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                         const float* oz, int64_t np, float mass, double c_poisson, const float* ux,
                         const float* uy, const float* uz, double scale, float* xbar, float* ybar,
                         float* zbar) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, ux, uy, uz, xbar, ybar, zbar}));
    PM_TRY(set_device(plan->p));
    const float* u[3] = {ux, uy, uz};
    float* xb[3] = {xbar, ybar, zbar};
    return adjoint_force_f32(plan->p, cell, ox, oy, oz, np, mass, c_poisson, u, scale, xb);
}

int pm_step_adjoint_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                        const float* oz, int64_t np, float mass, double c_poisson, double c_kick, double dt,
                        float* xbar, float* ybar, float* zbar, float* vxbar, float* vybar, float* vzbar) {
    PM_TRY(check_plan(plan, PM_FP32));
    PM_TRY(check_np(np, {cell, ox, oy, oz, xbar, ybar, zbar, vxbar, vybar, vzbar}));
    PM_TRY(set_device(plan->p));
    Plan& p = plan->p;
    float* vb[3] = {vxbar, vybar, vzbar};
    float* xb[3] = {xbar, ybar, zbar};
    const float* xbc[3] = {xbar, ybar, zbar};
    const float* vbc[3] = {vxbar, vybar, vzbar};
    if (dt != 0.0) PM_TRY(axpy3_f32(p, vb, xbc, dt, np));  // x' = x + dt v'  =>  vbar' += dt xbar
    if (c_kick == 0.0) return PM_OK;
    return adjoint_force_f32(p, cell, ox, oy, oz, np, mass, c_poisson, vbc, c_kick, xb);
}

// ------------------------------------------------------- FP64 reductions

static int reduce_args(pm_plan* plan, int precision, const void* vx, const void* vy, const void* vz, int64_t np,
                       const double* out) {
    PM_TRY(check_plan(plan, precision));
    if (!out) return fail(PM_ERR_ARG, "out is NULL");
    if (np < 0) return fail(PM_ERR_ARG, "np must be >= 0");
    if ((vx || vy || vz) && !(vx && vy && vz)) return fail(PM_ERR_ARG, "give all three velocity arrays or none");
    return set_device(plan->p);
}

int pm_reduce_f32(pm_plan* plan, const float* mesh, const float* vx, const float* vy, const float* vz,
                  int64_t np, double mass, double* out) {
    PM_TRY(reduce_args(plan, PM_FP32, vx, vy, vz, np, out));
    return reduce_conserved<float>(plan->p, mesh, vx, vy, vz, vx ? np : 0, mass, out);
}

int pm_reduce_f64(pm_plan* plan, const double* mesh, const double* vx, const double* vy, const double* vz,
                  int64_t np, double mass, double* out) {
    PM_TRY(reduce_args(plan, PM_FP64, vx, vy, vz, np, out));
    return reduce_conserved<double>(plan->p, mesh, vx, vy, vz, vx ? np : 0, mass, out);
}

// ------------------------------------------------------------------- ICs

int pm_ic_zeldovich(int ng, int nrow, double n_s, double rms_cells, uint64_t seed,
                    double vel_factor, double* x, double* y, double* z, double* vx, double* vy,
                    double* vz, void* stream) {
    if (!fft_size_supported(nrow)) return fail(PM_ERR_SIZE, "nrow must be a mesh size pm_plan_create takes");
    if (ng < 1) return fail(PM_ERR_ARG, "ng must be positive");
    if (!(rms_cells >= 0.0) || !std::isfinite(n_s)) return fail(PM_ERR_ARG, "bad spectrum parameters");
    PM_TRY(check_np(1, {x, y, z, vx, vy, vz}));
    pm_plan* plan = nullptr;
    PM_TRY(plan_create(nrow, PM_FP64, PM_GREEN_DISCRETE, 2, stream, &plan));
    const int rc = ic_zeldovich(plan->p, n_s, rms_cells, seed, vel_factor, ng, x, y, z, vx, vy, vz);
    pm_plan_destroy(plan);
    return rc;
}

}  // extern "C"
