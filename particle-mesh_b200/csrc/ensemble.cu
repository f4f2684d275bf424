// Batched ensemble of independent periodic boxes (FP32 split positions).
//
// No counterpart in the reference, which advances one box.  Boxes are grouped
// into size classes (same ng); each class is one batch: its meshes lie back to
// back and every kernel of the step (binning, the deposit - fused with the z
// R2C pass for power-of-two sizes -, the FFT passes with the Green multiply,
// gather + kick + drift) covers all boxes of the class in one launch.  Classes
// run on their own streams; a whole KDK run is captured once into a CUDA graph
// with one branch per class and replayed.  The shape of the strided FFT
// passes (column-tile width and radix split) is chosen per class by timing
// the candidates (autotune), optionally cached in a text file keyed by GPU
// name, mesh size, Green kind and gradient order (the analogue of the
// reference's FFTW wisdom file, src/fft/fftw/fft.cpp:28-49).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "pm_internal.cuh"

namespace pmb {

struct EnsembleClass {
    int ng = 0;
    std::vector<int> boxes;
    pm_plan* plan = nullptr;
    float* mesh = nullptr;
    long long* d_pbeg = nullptr;
    long long* d_pend = nullptr;
    float* d_mass = nullptr;
    int64_t np = 0;
    cudaEvent_t done = nullptr;
};

}  // namespace pmb

struct pm_ensemble {
    bool own_stream = false;
    int nbox = 0;
    int64_t np_total = 0;
    std::vector<pmb::EnsembleClass> classes;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    size_t bytes = 0;
    // cached graph of a KDK run and the arguments it was captured with
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key_ptrs;
    double key_cp = 0, key_dt = 0;
    int key_steps = -1;
    size_t graph_nodes = 0;
};

namespace pmb {

namespace {

void release_ensemble(pm_ensemble* e) {
    if (e->exec) cudaGraphExecDestroy(e->exec);
    for (auto& c : e->classes) {
        if (c.plan) {
            cudaStream_t s = c.plan->p.stream;
            pm_plan_destroy(c.plan);
            if (s) cudaStreamDestroy(s);
        }
        if (c.mesh) cudaFree(c.mesh);
        if (c.d_pbeg) cudaFree(c.d_pbeg);
        if (c.d_pend) cudaFree(c.d_pend);
        if (c.d_mass) cudaFree(c.d_mass);
        if (c.done) cudaEventDestroy(c.done);
    }
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

std::string gpu_name() {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "unknown";
    std::string s = prop.name;
    for (char& ch : s)
        if (ch == ' ') ch = '_';
    return s;
}

// Tune cache lines: "<gpu> <ng> <green> <order> <tk> <rv>" (tile width and
// radix split; a line without <rv> means the default split).
using TuneCache = std::map<std::string, std::pair<int, int>>;

TuneCache read_cache(const char* path) {
    TuneCache m;
    if (!path) return m;
    FILE* f = std::fopen(path, "r");
    if (!f) return m;
    char line[512], gpu[256];
    while (std::fgets(line, sizeof line, f)) {
        int ng, gk, go, tk, rv = 0;
        const int n = std::sscanf(line, "%255s %d %d %d %d %d", gpu, &ng, &gk, &go, &tk, &rv);
        if (n < 5) continue;
        m[std::string(gpu) + " " + std::to_string(ng) + " " + std::to_string(gk) + " " + std::to_string(go)] = {tk, rv};
    }
    std::fclose(f);
    return m;
}

void write_cache(const char* path, const TuneCache& m) {
    if (!path) return;
    FILE* f = std::fopen(path, "w");
    if (!f) return;
    for (auto& kv : m) std::fprintf(f, "%s %d %d\n", kv.first.c_str(), kv.second.first, kv.second.second);
    std::fclose(f);
}

int enqueue_step(pm_ensemble* e, EnsembleClass& c, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                 float* vy, float* vz, double c_poisson, double c_kick, double dt) {
    Plan& p = c.plan->p;
    const int nbox = (int)c.boxes.size();
    int rc;
    if (zcol_supported(c.ng)) {  // deposit fused with the z R2C pass, as in pm_step_f32
        rc = deposit_zr2c_f32_batch(p, cell, ox, oy, oz, c.d_pbeg, c.d_pend, nbox, c.np, c.d_mass, c.mesh);
        if (rc == PM_OK) rc = poisson_after_z_f32(p, c.mesh, c_poisson, nbox);
    } else {
        rc = deposit_f32_tiles_batch(p, cell, ox, oy, oz, c.d_pbeg, c.d_pend, nbox, c.np, c.d_mass, c.mesh);
        if (rc == PM_OK) rc = poisson_fused<float>(p, c.mesh, c_poisson, nbox);
    }
    if (rc == PM_OK)
        rc = kick_drift_f32_batch(p, c.mesh, cell, ox, oy, oz, vx, vy, vz, c.d_pbeg, c.d_pend, nbox, c.np, c_kick,
                                  dt);
    (void)e;
    return rc;
}

// Fork from the ensemble stream, run `body` on each class stream, join.
template <typename F>
int fork_join(pm_ensemble* e, F body) {
    PMB_CUDA_CHECK(cudaEventRecord(e->fork, e->stream));
    for (auto& c : e->classes) {
        PMB_CUDA_CHECK(cudaStreamWaitEvent(c.plan->p.stream, e->fork, 0));
        const int rc = body(c);
        if (rc != PM_OK) return rc;
        PMB_CUDA_CHECK(cudaEventRecord(c.done, c.plan->p.stream));
        PMB_CUDA_CHECK(cudaStreamWaitEvent(e->stream, c.done, 0));
    }
    return PM_OK;
}

std::string tune_key(const EnsembleClass& c) {
    const Plan& p = c.plan->p;
    return gpu_name() + " " + std::to_string(c.ng) + " " + std::to_string(p.green_kind) + " " +
           std::to_string(p.grad_order);
}

// A lattice of particles per box for the tuner: particle i of a box of ng^3
// cells sits in cell (i / ng^2, i / ng, i) mod ng with a fixed in-cell offset
// (a hash of i spread over [0.25, 0.75)), at rest.
__global__ void k_tune_lattice(uint32_t* __restrict__ cell, float* __restrict__ ox, float* __restrict__ oy,
                               float* __restrict__ oz, float* __restrict__ vx, float* __restrict__ vy,
                               float* __restrict__ vz, const long long* __restrict__ pbeg,
                               const long long* __restrict__ pend, int ng) {
    const long long lo = pbeg[blockIdx.y], hi = pend[blockIdx.y];
    for (long long p = lo + blockIdx.x * (long long)blockDim.x + threadIdx.x; p < hi;
         p += (long long)gridDim.x * blockDim.x) {
        const long long i = p - lo;
        const uint32_t x = (uint32_t)((i / ((long long)ng * ng)) % ng), y = (uint32_t)((i / ng) % ng),
                       z = (uint32_t)(i % ng);
        cell[p] = (x << 20) | (y << 10) | z;
        uint32_t h = (uint32_t)i * 2654435761u;
        ox[p] = 0.25f + 0.5f * (float)((h >> 8) & 1023u) / 1024.0f;
        h = h * 2654435761u + 12345u;
        oy[p] = 0.25f + 0.5f * (float)((h >> 8) & 1023u) / 1024.0f;
        h = h * 2654435761u + 12345u;
        oz[p] = 0.25f + 0.5f * (float)((h >> 8) & 1023u) / 1024.0f;
        vx[p] = vy[p] = vz[p] = 0.0f;
    }
}

// Median time of `reps` whole steps of every class (deposit, Poisson solve,
// gather + kick + drift on the tuner's lattice particles; c_kick = 0 and a
// tiny dt, so every rep does the same work), the classes on their own
// streams forked from and joined to the ensemble stream -- concurrently, as
// the captured graph runs them.
int time_steps(pm_ensemble* e, uint32_t* cell, float* f[6], int reps, cudaEvent_t a, cudaEvent_t b, float* out) {
    std::vector<float> ts;
    for (int r = 0; r < reps; ++r) {
        PMB_CUDA_CHECK(cudaEventRecord(a, e->stream));
        const int rc = fork_join(e, [&](EnsembleClass& c) {
            return enqueue_step(e, c, cell, f[0], f[1], f[2], f[3], f[4], f[5], 1.0, 0.0, 1e-6);
        });
        if (rc != PM_OK) return rc;
        PMB_CUDA_CHECK(cudaEventRecord(b, e->stream));
        PMB_CUDA_CHECK(cudaEventSynchronize(b));
        float ms = 0.f;
        PMB_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
        ts.push_back(ms);
    }
    std::nth_element(ts.begin(), ts.begin() + ts.size() / 2, ts.end());
    *out = ts[ts.size() / 2];
    return PM_OK;
}

// Shapes of the strided FFT passes (column-tile width x radix split) per
// class.  Classes found in the cache take the cached shape; the others (FP32
// power-of-two or mixed-radix ng <= 128) are tuned by coordinate descent: two
// rounds over the classes, each trying every candidate of one class while the
// others keep their current shape, scored by the median of 21 concurrent whole
// steps of all classes on a lattice of particles (temporary device arrays of
// the ensemble's particle count, freed before returning).  The shape of one
// class changes the time of the others: their kernels share the SMs.
int tune_shapes(pm_ensemble* e, TuneCache& cache, bool measure) {
    std::vector<EnsembleClass*> todo;
    for (auto& c : e->classes) {
        Plan& p = c.plan->p;
        auto it = cache.find(tune_key(c));
        if (it != cache.end() && tk_variant_supported(c.ng, PM_FP32, it->second.first) &&
            radix_variant_supported(c.ng, PM_FP32, it->second.second)) {
            p.tk = it->second.first;
            p.rv = it->second.second;
        } else if (c.ng <= 128) {
            todo.push_back(&c);
        }
    }
    if (!measure || todo.empty()) return PM_OK;
    const int64_t np = e->np_total > 0 ? e->np_total : 1;
    uint32_t* cell = nullptr;
    float* fbuf = nullptr;
    if (cudaMalloc(&cell, (size_t)np * 4) != cudaSuccess || cudaMalloc(&fbuf, (size_t)np * 24) != cudaSuccess) {
        cudaGetLastError();
        if (cell) cudaFree(cell);
        return fail(PM_ERR_NOMEM, "autotune: temporary particle arrays");
    }
    float* f[6];
    for (int a = 0; a < 6; ++a) f[a] = fbuf + (size_t)a * np;
    int rc = PM_OK;
    for (auto& c : e->classes) {
        const Plan& p = c.plan->p;
        k_tune_lattice<<<dim3(grid_for(p, (long long)c.ng * c.ng * c.ng, 256, 2), (unsigned)c.boxes.size()), 256, 0,
                         p.stream>>>(cell, f[0], f[1], f[2], f[3], f[4], f[5], c.d_pbeg, c.d_pend, c.ng);
        if (cudaGetLastError() != cudaSuccess) rc = fail(PM_ERR_CUDA, "autotune: lattice fill");
    }
    cudaEvent_t a = nullptr, b = nullptr;
    if (rc == PM_OK && (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess))
        rc = fail(PM_ERR_CUDA, "autotune: events");
    float t = 0.f;
    if (rc == PM_OK) rc = time_steps(e, cell, f, 3, a, b, &t);  // warm-up
    for (int round = 0; round < 2 && rc == PM_OK; ++round) {
        for (EnsembleClass* c : todo) {
            Plan& p = c->plan->p;
            int best_tk = p.tk, best_rv = p.rv;
            float best = 0.f;
            rc = time_steps(e, cell, f, 21, a, b, &best);
            for (int rv : {0, 1}) {
                if (rc != PM_OK || !radix_variant_supported(c->ng, PM_FP32, rv)) continue;
                for (int tk : {0, 8, 16, 32}) {
                    if (rc != PM_OK || !tk_variant_supported(c->ng, PM_FP32, tk) || (tk == best_tk && rv == best_rv))
                        continue;
                    p.tk = tk;
                    p.rv = rv;
                    rc = time_steps(e, cell, f, 21, a, b, &t);
                    if (rc == PM_OK && t < best) {
                        best = t;
                        best_tk = tk;
                        best_rv = rv;
                    }
                }
            }
            p.tk = best_tk;
            p.rv = best_rv;
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaDeviceSynchronize();
    cudaFree(cell);
    cudaFree(fbuf);
    if (rc != PM_OK) return rc;
    for (EnsembleClass* c : todo) cache[tune_key(*c)] = {c->plan->p.tk, c->plan->p.rv};
    return PM_OK;
}

}  // namespace
}  // namespace pmb

using namespace pmb;

extern "C" {

int pm_ensemble_create(int nbox, const int* ng, const int64_t* np, const float* mass, int green_kind,
                       int grad_order, int autotune, const char* tune_cache, void* stream, pm_ensemble** out) {
    if (!out) return fail(PM_ERR_ARG, "output pointer is NULL");
    *out = nullptr;
    if (nbox <= 0 || !ng || !np || !mass) return fail(PM_ERR_ARG, "need nbox > 0 and ng, np, mass arrays");
    for (int b = 0; b < nbox; ++b) {
        if (!fft_size_supported(ng[b])) return fail(PM_ERR_SIZE, "ensemble box mesh size not supported");
        if (np[b] < 0) return fail(PM_ERR_ARG, "negative particle count");
    }
    pm_ensemble* e = new (std::nothrow) pm_ensemble();
    if (!e) return fail(PM_ERR_NOMEM, "host allocation failed");
    e->nbox = nbox;
    e->stream = static_cast<cudaStream_t>(stream);
    if (!e->stream) {  // graphs cannot be captured on the legacy default stream
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete e;
            return fail(PM_ERR_CUDA, "stream creation failed");
        }
        e->own_stream = true;
    }
    std::vector<int64_t> off(nbox + 1, 0);
    for (int b = 0; b < nbox; ++b) off[b + 1] = off[b] + np[b];
    e->np_total = off[nbox];
    std::map<int, std::vector<int>> groups;
    for (int b = 0; b < nbox; ++b) groups[ng[b]].push_back(b);
    int rc = PM_OK;
    if (cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(PM_ERR_CUDA, "event creation failed");
    for (auto& g : groups) {
        if (rc != PM_OK) break;
        EnsembleClass c;
        c.ng = g.first;
        c.boxes = g.second;
        cudaStream_t cs = nullptr;
        if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
            rc = fail(PM_ERR_CUDA, "stream creation failed");
            break;
        }
        rc = pm_plan_create(c.ng, PM_FP32, green_kind, grad_order, cs, &c.plan);
        if (rc != PM_OK) {
            cudaStreamDestroy(cs);
            break;
        }
        const size_t nb = c.boxes.size();
        std::vector<long long> pb(nb), pe(nb);
        std::vector<float> m(nb);
        for (size_t i = 0; i < nb; ++i) {
            pb[i] = off[c.boxes[i]];
            pe[i] = off[c.boxes[i] + 1];
            m[i] = mass[c.boxes[i]];
            c.np += np[c.boxes[i]];
        }
        const size_t mb = mesh_elems(c.ng) * nb * sizeof(float);
        if (cudaMalloc(&c.mesh, mb) != cudaSuccess || cudaMalloc(&c.d_pbeg, nb * 8) != cudaSuccess ||
            cudaMalloc(&c.d_pend, nb * 8) != cudaSuccess || cudaMalloc(&c.d_mass, nb * 4) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            e->classes.push_back(c);
            rc = fail(PM_ERR_NOMEM, "ensemble allocation failed");
            break;
        }
        cudaMemcpy(c.d_pbeg, pb.data(), nb * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(c.d_pend, pe.data(), nb * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(c.d_mass, m.data(), nb * 4, cudaMemcpyHostToDevice);
        // scratch for the batched binning, allocated now so that steps (and
        // graph captures) never allocate
        rc = tile_scratch_ensure(c.plan->p, c.np > 0 ? c.np : 1, (int)nb);
        e->bytes += mb + nb * 20 + c.plan->p.bytes;
        e->classes.push_back(c);
    }
    if (rc == PM_OK) {
        auto cache = read_cache(tune_cache);
        const size_t before = cache.size();
        rc = tune_shapes(e, cache, autotune != 0);
        if (rc == PM_OK && cache.size() != before) write_cache(tune_cache, cache);
        if (rc == PM_OK && cudaDeviceSynchronize() != cudaSuccess) rc = fail(PM_ERR_CUDA, "autotune failed");
    }
    if (rc != PM_OK) {
        release_ensemble(e);
        return rc;
    }
    *out = e;
    return PM_OK;
}

int pm_ensemble_destroy(pm_ensemble* e) {
    if (!e) return PM_OK;
    cudaStreamSynchronize(e->stream);
    for (auto& c : e->classes)
        if (c.plan) cudaStreamSynchronize(c.plan->p.stream);
    release_ensemble(e);
    return PM_OK;
}

int pm_ensemble_sync(pm_ensemble* e) {
    if (!e) return fail(PM_ERR_ARG, "ensemble is NULL");
    PMB_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return PM_OK;
}

int pm_ensemble_info(const pm_ensemble* e, int* nclasses, int* class_ng, int* class_nbox, int* class_tk,
                     int* class_radix, size_t* device_bytes, size_t* graph_nodes) {
    if (!e) return fail(PM_ERR_ARG, "ensemble is NULL");
    if (nclasses) *nclasses = (int)e->classes.size();
    for (size_t i = 0; i < e->classes.size(); ++i) {
        const Plan& p = e->classes[i].plan->p;
        if (class_ng) class_ng[i] = e->classes[i].ng;
        if (class_nbox) class_nbox[i] = (int)e->classes[i].boxes.size();
        if (class_tk) class_tk[i] = p.tk;
        if (class_radix) class_radix[i] = strided_radix1(p.ng, p.rv);
    }
    if (device_bytes) *device_bytes = e->bytes;
    if (graph_nodes) *graph_nodes = e->graph_nodes;
    return PM_OK;
}

int pm_ensemble_step_f32(pm_ensemble* e, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                         float* vz, double c_poisson, double c_kick, double dt) {
    if (!e) return fail(PM_ERR_ARG, "ensemble is NULL");
    if (e->np_total > 0 && (!cell || !ox || !oy || !oz || !vx || !vy || !vz))
        return fail(PM_ERR_ARG, "NULL particle array");
    return fork_join(e, [&](EnsembleClass& c) {
        return enqueue_step(e, c, cell, ox, oy, oz, vx, vy, vz, c_poisson, c_kick, dt);
    });
}

int pm_ensemble_run_f32(pm_ensemble* e, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                        float* vz, double c_poisson, double dt, int steps) {
    if (!e) return fail(PM_ERR_ARG, "ensemble is NULL");
    if (steps < 0) return fail(PM_ERR_ARG, "negative step count");
    if (e->np_total > 0 && (!cell || !ox || !oy || !oz || !vx || !vy || !vz))
        return fail(PM_ERR_ARG, "NULL particle array");
    std::vector<const void*> ptrs = {cell, ox, oy, oz, vx, vy, vz};
    const bool hit = e->exec && e->key_ptrs == ptrs && e->key_cp == c_poisson && e->key_dt == dt &&
                     e->key_steps == steps;
    if (!hit) {
        if (e->exec) cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
        for (auto& c : e->classes) c.plan->p.timers->on = false;  // no timing events inside the graph
        PMB_CUDA_CHECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        // KDK with merged half kicks: steps + 1 force evaluations
        int rc = fork_join(e, [&](EnsembleClass& c) {
            for (int s = 0; s <= steps; ++s) {
                const double ck = (s == 0 || s == steps) ? 0.5 * dt : dt, dd = s < steps ? dt : 0.0;
                const int r = enqueue_step(e, c, cell, ox, oy, oz, vx, vy, vz, c_poisson, ck, dd);
                if (r != PM_OK) return r;
            }
            return PM_OK;
        });
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
        if (rc != PM_OK) {
            if (graph) cudaGraphDestroy(graph);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        cudaGraphGetNodes(graph, nullptr, &e->graph_nodes);
        const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            e->exec = nullptr;
            return cuda_fail(ie, "cudaGraphInstantiate");
        }
        e->key_ptrs = ptrs;
        e->key_cp = c_poisson;
        e->key_dt = dt;
        e->key_steps = steps;
    }
    PMB_CUDA_CHECK(cudaGraphLaunch(e->exec, e->stream));
    return PM_OK;
}

}  // extern "C"
