// x-slab decomposition of one periodic mesh over several ranks (one GPU
// each): the reference's own parallel layout.  The reference splits the
// particles and the mesh into cubes, sends each cube with its +1 ghost planes
// to the owners of FFT x-slabs (src/decomp/slab/transpose_slab.cpp:3-39),
// folds the ghosts there (reorder_slab.cpp:43-68), lets FFTW-MPI transpose
// the spectrum (src/fft/fftw/fft.cpp:16, 96-97, FFTW_MPI_TRANSPOSED_OUT/IN),
// and sends the potential back with -1/+2 ghost planes
// (reorder_slab_back.cpp:37-49, transpose_slab_back.cpp:3-49).  Here the
// particles live on the slab that owns their x plane, so:
//
//   deposit      the slab's particles, fused with the z R2C, into its own
//                planes plus one ghost plane (the +1 corners of its last
//                plane), which the next slab adds to its first plane;
//   y forward    over the own planes, stored as rows [ky][x][kz] of the
//                send buffer so that each destination's ky range is
//                contiguous;
//   (all-to-all) the global transpose;
//   x + Green    x lines read across the received blocks [rank][kyl][x][kz],
//                x forward, Green, x inverse, written into the same layout
//                of the send buffer (block d back to rank d);
//   (all-to-all) the transpose back;
//   y inverse    read from the received rows [ky][x][kz], written into
//                the own planes; z C2R over them;
//   (halo)       two planes from the previous slab, three from the next
//                (the 4-point stencil reaches x - 2 .. x + 3);
//   gather + kick + drift, then particles that left the slab migrate to
//   their new owner (new: the reference never moves particles).
//
// The exchanges belong to the caller (NCCL through torch.distributed, or
// copies between slabs emulated on one GPU); this file holds the per-slab
// kernels and buffers.
#include <cstring>
#include <new>
#include <vector>

#include "pm_internal.cuh"

namespace pmb {

namespace {

// plane += ghost over one padded plane of ng (ng + 2) floats (float2 pairs).
__global__ void k_fold_plane(float2* __restrict__ plane, const float2* __restrict__ ghost, long long n2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x) {
        const float2 a = plane[i], b = ghost[i];
        plane[i] = make_float2(a.x + b.x, a.y + b.y);
    }
}

struct Words {
    uint32_t* a[8];
};

// packed[i][w] = arrays[w][perm[i]]: the particles in destination order,
// W 32-bit words each.
__global__ void k_pack_words(const uint32_t* __restrict__ perm, long long n, Words src, int nw,
                             uint32_t* __restrict__ packed) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t p = __ldg(perm + i);
        for (int w = 0; w < nw; ++w) packed[i * nw + w] = src.a[w][p];
    }
}

// arrays[w][at + i] = packed[i][w].
__global__ void k_unpack_words(const uint32_t* __restrict__ packed, long long n, Words dst, int nw, long long at) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        for (int w = 0; w < nw; ++w) dst.a[w][at + i] = __ldg(packed + i * nw + w);
}

}  // namespace

struct Slab {
    pm_plan* plan = nullptr;  // FP32 plan of the whole mesh: tables, stream, timers, binning scratch
    int ng = 0, nranks = 1, rank = 0, nx = 0, x0 = 0, nyl = 0, ky0 = 0;
    float* buf = nullptr;      // [nx + 6][ng][ng + 2]: planes 0-1 lower halo, 2..nx+1 own, nx+2.. ghost / upper halo
    float2* send = nullptr;    // nx ng H complex
    float2* recv = nullptr;    // nx ng H complex
    size_t bytes = 0;
    size_t plane_floats() const { return (size_t)ng * (ng + 2); }
    float* own() const { return buf + 2 * plane_floats(); }
    long long rows() const { return (long long)nx * ng; }
};

static void slab_release(Slab& s) {
    if (s.buf) cudaFree(s.buf);
    if (s.send) cudaFree(s.send);
    if (s.recv) cudaFree(s.recv);
    if (s.plan) pm_plan_destroy(s.plan);
    s.buf = nullptr;
    s.send = s.recv = nullptr;
    s.plan = nullptr;
}

// One rank's pencil of a Px x Py decomposition: x in [x0, x0 + nx), y in
// [y0, y0 + ny), all z.  The spectrum is split into Py kz chunks
// [kb(c), kb(c + 1)), kb(c) = c H / Py (H = ng/2 + 1), for the y stage and
// into Px ky chunks of yc = ng / Px for the x stage.
struct Pencil {
    pm_plan* plan = nullptr;
    int ng = 0, px = 1, py = 1, rank = 0, rx = 0, ry = 0, nx = 0, ny = 0, x0 = 0, y0 = 0, yc = 0, h = 0;
    float* halo = nullptr;  // [nx + 5][ny + 5][ng + 2]
    float2* own = nullptr;  // [nx][ny][h]
    float2* send = nullptr;
    float2* recv = nullptr;
    long long xfer = 0;  // complex entries of each of send / recv
    size_t bytes = 0;
    int kb(int c) const { return (int)((long long)c * h / py); }
    int hc(int c) const { return kb(c + 1) - kb(c); }
    long long yoff(int c) const { return (long long)nx * ny * kb(c); }  // y-stage block c at nx ny kb(c)
    float2* halo_c() const { return reinterpret_cast<float2*>(halo); }
    long long hrow(int xl, int yl) const { return ((long long)xl * (ny + 5) + yl) * h; }  // complex offset
};

static void pencil_release(Pencil& q) {
    for (void* b : {(void*)q.halo, (void*)q.own, (void*)q.send, (void*)q.recv})
        if (b) cudaFree(b);
    if (q.plan) pm_plan_destroy(q.plan);
    q = Pencil{};
}

namespace {
__global__ void k_add_rows(float* __restrict__ dst, long long dstride, const float* __restrict__ src, int nrows,
                           int rowlen) {
    const long long n = (long long)nrows * rowlen;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / rowlen, c = e - r * rowlen;
        dst[r * dstride + c] += src[e];
    }
}
}  // namespace

}  // namespace pmb

struct pm_slab {
    pmb::Slab s;
};

struct pm_pencil {
    pmb::Pencil q;
};

using namespace pmb;

#define PM_TRY_S(expr)                \
    do {                              \
        int _rc = (expr);             \
        if (_rc != PM_OK) return _rc; \
    } while (0)

static int slab_ok(const pm_slab* slab) {
    if (!slab || !slab->s.plan) return fail(PM_ERR_ARG, "slab is NULL");
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail(PM_ERR_CUDA, "cudaGetDevice failed");
    if (cur != slab->s.plan->p.device) PMB_CUDA_CHECK(cudaSetDevice(slab->s.plan->p.device));
    return PM_OK;
}

extern "C" {

int pm_slab_create(int ng, int nranks, int rank, int green_kind, int grad_order, void* stream, pm_slab** out) {
    if (!out) return fail(PM_ERR_ARG, "output pointer is NULL");
    *out = nullptr;
    if (!(ng >= 32 && ng <= 1024 && (ng & (ng - 1)) == 0))
        return fail(PM_ERR_SIZE, "the slab path needs a power-of-two ng in [32, 1024]");
    if (nranks < 1 || (nranks & (nranks - 1)) != 0 || ng % (4 * nranks) != 0)
        return fail(PM_ERR_SIZE, "nranks must be a power of two with ng / nranks a multiple of 4");
    if (rank < 0 || rank >= nranks) return fail(PM_ERR_ARG, "rank out of range");
    pm_slab* slab = new (std::nothrow) pm_slab();
    if (!slab) return fail(PM_ERR_NOMEM, "host allocation failed");
    Slab& s = slab->s;
    s.ng = ng;
    s.nranks = nranks;
    s.rank = rank;
    s.nx = s.nyl = ng / nranks;
    s.x0 = s.ky0 = rank * s.nx;
    int rc = plan_create_internal(ng, PM_FP32, green_kind, grad_order, stream, &s.plan);
    if (rc != PM_OK) {
        delete slab;
        return rc;
    }
    const size_t bufb = (size_t)(s.nx + 6) * s.plane_floats() * sizeof(float);
    const size_t xfer = (size_t)s.rows() * (ng / 2 + 1) * sizeof(float2);
    if (cudaMalloc(&s.buf, bufb) != cudaSuccess || cudaMalloc(&s.send, xfer) != cudaSuccess ||
        cudaMalloc(&s.recv, xfer) != cudaSuccess || cudaMemset(s.buf, 0, bufb) != cudaSuccess) {
        cudaGetLastError();
        slab_release(s);
        delete slab;
        return fail(PM_ERR_NOMEM, "slab buffer allocation failed");
    }
    s.bytes = bufb + 2 * xfer;
    *out = slab;
    return PM_OK;
}

int pm_slab_destroy(pm_slab* slab) {
    if (!slab) return PM_OK;
    if (slab->s.plan) {
        cudaSetDevice(slab->s.plan->p.device);
        cudaStreamSynchronize(slab->s.plan->p.stream);
    }
    slab_release(slab->s);
    delete slab;
    return PM_OK;
}

int pm_slab_info(const pm_slab* slab, int* nx, int* x0, size_t* plane_floats, void** buf, void** send, void** recv,
                 size_t* xfer_floats, size_t* device_bytes) {
    if (!slab || !slab->s.plan) return fail(PM_ERR_ARG, "slab is NULL");
    const Slab& s = slab->s;
    if (nx) *nx = s.nx;
    if (x0) *x0 = s.x0;
    if (plane_floats) *plane_floats = s.plane_floats();
    if (buf) *buf = s.buf;
    if (send) *send = s.send;
    if (recv) *recv = s.recv;
    if (xfer_floats) *xfer_floats = (size_t)s.rows() * (s.ng + 2);
    if (device_bytes) *device_bytes = s.bytes + s.plan->p.bytes;
    return PM_OK;
}

int pm_slab_plan(pm_slab* slab, pm_plan** plan) {
    if (!slab || !plan) return fail(PM_ERR_ARG, "NULL argument");
    *plan = slab->s.plan;
    return PM_OK;
}

int pm_slab_deposit_f32(pm_slab* slab, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                        int64_t np, float mass) {
    PM_TRY_S(slab_ok(slab));
    if (np < 0) return fail(PM_ERR_ARG, "negative particle count");
    if (np > 0 && (!cell || !ox || !oy || !oz)) return fail(PM_ERR_ARG, "NULL particle array");
    Slab& s = slab->s;
    return slab_deposit_zr2c_f32(s.plan->p, s.x0, s.nx, cell, ox, oy, oz, np, mass, s.own());
}

int pm_slab_fold_f32(pm_slab* slab, const float* ghost) {
    PM_TRY_S(slab_ok(slab));
    if (!ghost) return fail(PM_ERR_ARG, "ghost is NULL");
    Slab& s = slab->s;
    const Plan& p = s.plan->p;
    const long long n2 = (long long)s.plane_floats() / 2;
    {
        Timed t(p, ST_DEPOSIT);
        k_fold_plane<<<grid_for(p, n2, 256, 4), 256, 0, p.stream>>>(reinterpret_cast<float2*>(s.own()),
                                                                    reinterpret_cast<const float2*>(ghost), n2);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// The row permutations of the transposes are folded into the FFT passes'
// loads and stores: the y forward writes the rows [ky][x][kz] of `send`, the
// x + Green pass reads the received blocks and writes the ones to send back,
// the y inverse reads the received rows (no separate copy of the spectrum).
int pm_slab_forward_f32(pm_slab* slab) {
    PM_TRY_S(slab_ok(slab));
    Slab& s = slab->s;
    return slab_fft_forward_y_f32(s.plan->p, s.own(), reinterpret_cast<float*>(s.send), s.nx);
}

int pm_slab_xgreen_f32(pm_slab* slab, double c_poisson) {
    PM_TRY_S(slab_ok(slab));
    Slab& s = slab->s;
    return slab_fft_xgreen_f32(s.plan->p, reinterpret_cast<const float*>(s.recv), reinterpret_cast<float*>(s.send),
                               c_poisson, s.nx, s.ky0);
}

int pm_slab_backward_f32(pm_slab* slab) {
    PM_TRY_S(slab_ok(slab));
    Slab& s = slab->s;
    return slab_fft_backward_f32(s.plan->p, reinterpret_cast<const float*>(s.recv), s.own(), s.nx);
}

// Transposes by stores into the other ranks' memory: the y forward and the
// x + Green pass write each output row into the buffer of the rank that
// owns it (peer device pointers, e.g. from symmetric memory), at this rank's
// block; no collective moves the spectrum.  The caller separates the phases
// with a barrier across the ranks (every store done before a rank reads).
static int peer_map(const Slab& s, void* const* peers, int npeers, long long block, long long ps, int s0, int n,
                    PeerMap& po) {
    if (!peers || npeers != s.nranks) return fail(PM_ERR_ARG, "one peer buffer per rank expected");
    if (npeers > kMaxPeers) return fail(PM_ERR_SIZE, "at most 16 ranks for the peer-store transposes");
    for (int d = 0; d < npeers; ++d) {
        if (!peers[d]) return fail(PM_ERR_ARG, "NULL peer buffer");
        po.base[d] = static_cast<float2*>(peers[d]) + block;
    }
    int l = 0;
    while ((1 << l) < n) ++l;
    po.ps = ps;
    po.s0 = s0;
    po.sl = l;
    po.mask = n - 1;
    return PM_OK;
}

int pm_slab_forward_peers_f32(pm_slab* slab, void* const* peer_recv, int npeers) {
    PM_TRY_S(slab_ok(slab));
    Slab& s = slab->s;
    const int H = s.ng / 2 + 1;
    // row (ky, x) to rank ky / nyl, its block `rank`, at (ky mod nyl) nx + x
    PeerMap po;
    PM_TRY_S(peer_map(s, peer_recv, npeers, (long long)s.rank * s.nyl * s.nx * H, H, s.nx * H, s.nyl, po));
    return slab_fft_forward_peers_f32(s.plan->p, s.own(), po, s.nx);
}

int pm_slab_xgreen_peers_f32(pm_slab* slab, const void* recv, double c_poisson, void* const* peer_rows,
                             int npeers) {
    PM_TRY_S(slab_ok(slab));
    if (!recv) return fail(PM_ERR_ARG, "recv is NULL");
    Slab& s = slab->s;
    const int H = s.ng / 2 + 1;
    // line (kyl, kx) to rank kx / nx, row (ky0 + kyl) nx + kx mod nx of its rows [ky][x][kz]
    PeerMap po;
    PM_TRY_S(peer_map(s, peer_rows, npeers, (long long)s.ky0 * s.nx * H, (long long)s.nx * H, H, s.nx, po));
    return slab_fft_xgreen_peers_f32(s.plan->p, static_cast<const float*>(recv), po, c_poisson, s.nx, s.ky0);
}

int pm_slab_backward_rows_f32(pm_slab* slab, const void* rows) {
    PM_TRY_S(slab_ok(slab));
    if (!rows) return fail(PM_ERR_ARG, "rows is NULL");
    Slab& s = slab->s;
    return slab_fft_backward_f32(s.plan->p, static_cast<const float*>(rows), s.own(), s.nx);
}

int pm_slab_kick_drift_f32(pm_slab* slab, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                           float* vz, int64_t np, double c_kick, double dt) {
    PM_TRY_S(slab_ok(slab));
    if (np < 0) return fail(PM_ERR_ARG, "negative particle count");
    if (np > 0 && (!cell || !ox || !oy || !oz || !vx || !vy || !vz)) return fail(PM_ERR_ARG, "NULL particle array");
    Slab& s = slab->s;
    return slab_kick_drift_f32(s.plan->p, s.x0, s.nx, s.buf, cell, ox, oy, oz, vx, vy, vz, np, c_kick, dt);
}

int pm_slab_migrate_sort(pm_slab* slab, const uint32_t* cell, int64_t np, int64_t* counts) {
    PM_TRY_S(slab_ok(slab));
    if (np < 0 || !counts || (np > 0 && !cell)) return fail(PM_ERR_ARG, "bad migration arguments");
    if (np > (int64_t)0xffffffffll) return fail(PM_ERR_SIZE, "a slab holds at most 2^32 - 1 particles");
    Slab& s = slab->s;
    return slab_rank_sort(s.plan->p, s.nranks, s.nx, cell, np, counts);
}

int pm_slab_migrate_pack(pm_slab* slab, void* const* arrays, int narrays, int64_t np, uint32_t* packed) {
    PM_TRY_S(slab_ok(slab));
    if (!arrays || narrays < 1 || narrays > 8 || np < 0 || (np > 0 && !packed))
        return fail(PM_ERR_ARG, "bad pack arguments");
    Words w{};
    for (int a = 0; a < narrays; ++a) {
        w.a[a] = static_cast<uint32_t*>(arrays[a]);
        if (np > 0 && !w.a[a]) return fail(PM_ERR_ARG, "NULL particle array");
    }
    Slab& s = slab->s;
    const Plan& p = s.plan->p;
    if (np > s.plan->p.tiles.np_cap) return fail(PM_ERR_STATE, "pm_slab_migrate_sort must precede the pack");
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_SORT);
        k_pack_words<<<grid_for(p, np, 256, 4), 256, 0, p.stream>>>(p.tiles.perm, np, w, narrays, packed);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pm_slab_migrate_unpack(pm_slab* slab, const uint32_t* packed, int64_t n, void* const* arrays, int narrays,
                           int64_t at) {
    PM_TRY_S(slab_ok(slab));
    if (!arrays || narrays < 1 || narrays > 8 || n < 0 || at < 0 || (n > 0 && !packed))
        return fail(PM_ERR_ARG, "bad unpack arguments");
    Words w{};
    for (int a = 0; a < narrays; ++a) {
        w.a[a] = static_cast<uint32_t*>(arrays[a]);
        if (n > 0 && !w.a[a]) return fail(PM_ERR_ARG, "NULL particle array");
    }
    if (n == 0) return PM_OK;
    const Plan& p = slab->s.plan->p;
    {
        Timed t(p, ST_SORT);
        k_unpack_words<<<grid_for(p, n, 256, 4), 256, 0, p.stream>>>(packed, n, w, narrays, at);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// ------------------------------------------------------ CUDA IPC of buffers

int pm_ipc_export(const void* dev_ptr, void* handle) {
    if (!dev_ptr || !handle) return fail(PM_ERR_ARG, "NULL argument");
    cudaIpcMemHandle_t h;
    PMB_CUDA_CHECK(cudaIpcGetMemHandle(&h, const_cast<void*>(dev_ptr)));
    static_assert(sizeof(h) <= PM_IPC_HANDLE_BYTES, "IPC handle size");
    std::memset(handle, 0, PM_IPC_HANDLE_BYTES);
    std::memcpy(handle, &h, sizeof(h));
    return PM_OK;
}

int pm_ipc_open(const void* handle, void** dev_ptr) {
    if (!dev_ptr || !handle) return fail(PM_ERR_ARG, "NULL argument");
    *dev_ptr = nullptr;
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof(h));
    PMB_CUDA_CHECK(cudaIpcOpenMemHandle(dev_ptr, h, cudaIpcMemLazyEnablePeerAccess));
    return PM_OK;
}

int pm_ipc_close(void* dev_ptr) {
    if (!dev_ptr) return PM_OK;
    PMB_CUDA_CHECK(cudaIpcCloseMemHandle(dev_ptr));
    return PM_OK;
}

int pm_slab_check(pm_slab* slab) {
    if (!slab || !slab->s.plan) return fail(PM_ERR_ARG, "slab is NULL");
    return pm_plan_check(slab->s.plan);
}

// ------------------------------------------------------------- pencils

static int pencil_ok(const pm_pencil* pen) {
    if (!pen || !pen->q.plan) return fail(PM_ERR_ARG, "pencil is NULL");
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail(PM_ERR_CUDA, "cudaGetDevice failed");
    if (cur != pen->q.plan->p.device) PMB_CUDA_CHECK(cudaSetDevice(pen->q.plan->p.device));
    return PM_OK;
}

int pm_pencil_create(int ng, int px, int py, int rank, int green_kind, int grad_order, void* stream,
                     pm_pencil** out) {
    if (!out) return fail(PM_ERR_ARG, "output pointer is NULL");
    *out = nullptr;
    if (!(ng >= 32 && ng <= 1024 && (ng & (ng - 1)) == 0))
        return fail(PM_ERR_SIZE, "the pencil path needs a power-of-two ng in [32, 1024]");
    auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
    if (!pow2(px) || !pow2(py) || ng / px < 4 || ng / py < 4)
        return fail(PM_ERR_SIZE, "px and py must be powers of two with ng / px and ng / py at least 4");
    if (py > ng / 2 + 1) return fail(PM_ERR_SIZE, "py exceeds the kz planes of the half spectrum");
    if (rank < 0 || rank >= px * py) return fail(PM_ERR_ARG, "rank out of range");
    pm_pencil* pen = new (std::nothrow) pm_pencil();
    if (!pen) return fail(PM_ERR_NOMEM, "host allocation failed");
    Pencil& q = pen->q;
    q.ng = ng;
    q.px = px;
    q.py = py;
    q.rank = rank;
    q.rx = rank / py;
    q.ry = rank % py;
    q.nx = ng / px;
    q.ny = ng / py;
    q.x0 = q.rx * q.nx;
    q.y0 = q.ry * q.ny;
    q.yc = ng / px;
    q.h = ng / 2 + 1;
    int rc = plan_create_internal(ng, PM_FP32, green_kind, grad_order, stream, &q.plan);
    if (rc != PM_OK) {
        delete pen;
        return rc;
    }
    const int hcmax = (q.h + py - 1) / py;
    q.xfer = (long long)q.nx * ng * hcmax;
    const size_t haloB = (size_t)(q.nx + 5) * (q.ny + 5) * (ng + 2) * sizeof(float);
    const size_t ownB = (size_t)q.nx * q.ny * q.h * sizeof(float2), xB = (size_t)q.xfer * sizeof(float2);
    if (cudaMalloc(&q.halo, haloB) != cudaSuccess || cudaMalloc(&q.own, ownB) != cudaSuccess ||
        cudaMalloc(&q.send, xB) != cudaSuccess || cudaMalloc(&q.recv, xB) != cudaSuccess ||
        cudaMemset(q.halo, 0, haloB) != cudaSuccess) {
        cudaGetLastError();
        pencil_release(q);
        delete pen;
        return fail(PM_ERR_NOMEM, "pencil buffer allocation failed");
    }
    q.bytes = haloB + ownB + 2 * xB;
    *out = pen;
    return PM_OK;
}

int pm_pencil_destroy(pm_pencil* pen) {
    if (!pen) return PM_OK;
    if (pen->q.plan) {
        cudaSetDevice(pen->q.plan->p.device);
        cudaStreamSynchronize(pen->q.plan->p.stream);
    }
    pencil_release(pen->q);
    delete pen;
    return PM_OK;
}

int pm_pencil_info(const pm_pencil* pen, int* nx, int* ny, int* x0, int* y0, void** halo, void** send, void** recv,
                   size_t* xfer_floats, size_t* device_bytes) {
    if (!pen || !pen->q.plan) return fail(PM_ERR_ARG, "pencil is NULL");
    const Pencil& q = pen->q;
    if (nx) *nx = q.nx;
    if (ny) *ny = q.ny;
    if (x0) *x0 = q.x0;
    if (y0) *y0 = q.y0;
    if (halo) *halo = q.halo;
    if (send) *send = q.send;
    if (recv) *recv = q.recv;
    if (xfer_floats) *xfer_floats = (size_t)q.xfer * 2;
    if (device_bytes) *device_bytes = q.bytes + q.plan->p.bytes;
    return PM_OK;
}

int pm_pencil_plan(pm_pencil* pen, pm_plan** plan) {
    if (!pen || !plan) return fail(PM_ERR_ARG, "NULL argument");
    *plan = pen->q.plan;
    return PM_OK;
}

int pm_pencil_deposit_f32(pm_pencil* pen, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                          int64_t np, float mass) {
    PM_TRY_S(pencil_ok(pen));
    if (np < 0) return fail(PM_ERR_ARG, "negative particle count");
    if (np > 0 && (!cell || !ox || !oy || !oz)) return fail(PM_ERR_ARG, "NULL particle array");
    Pencil& q = pen->q;
    return pencil_deposit_f32(q.plan->p, q.x0, q.y0, q.nx, q.ny, cell, ox, oy, oz, np, mass, q.halo);
}

int pm_pencil_fold_f32(pm_pencil* pen, const float* xghost, const float* yghost, const float* corner) {
    PM_TRY_S(pencil_ok(pen));
    if (!xghost || !yghost || !corner) return fail(PM_ERR_ARG, "NULL ghost rows");
    Pencil& q = pen->q;
    const Plan& p = q.plan->p;
    const int rl = q.ng + 2;
    const long long row = rl, plane = (long long)(q.ny + 5) * rl;
    {
        Timed t(p, ST_DEPOSIT, 3);
        // x ghost: rows (2, 2..ny+1); y ghost: rows (2..nx+1, 2); corner: (2, 2)
        k_add_rows<<<grid_for(p, (long long)q.ny * rl, 256, 2), 256, 0, p.stream>>>(q.halo + 2 * plane + 2 * row, row,
                                                                                   xghost, q.ny, rl);
        k_add_rows<<<grid_for(p, (long long)q.nx * rl, 256, 2), 256, 0, p.stream>>>(q.halo + 2 * plane + 2 * row,
                                                                                   plane, yghost, q.nx, rl);
        k_add_rows<<<grid_for(p, rl, 256, 2), 256, 0, p.stream>>>(q.halo + 2 * plane + 2 * row, row, corner, 1, rl);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// own rows out of the halo buffer (with the -1 background) and the z R2C;
// then kz chunk c ([nx][ny][hc(c)]) to dst[c] (row strides ny hc(c), hc(c))
static int pencil_forward_to(Pencil& q, const std::vector<float2*>& dst) {
    const Plan& p = q.plan->p;
    const long long H = q.h, ny = q.ny, nx = q.nx;
    {
        Timed t(p, ST_SORT);
        // own rows into the compact buffer, with the density contrast's -1
        PM_TRY_S(pencil_copy3(p, q.halo_c() + q.hrow(2, 2), (ny + 5) * H, H, q.own, ny * H, H, q.nx, q.ny, q.h, 1.0f));
    }
    PM_TRY_S(pencil_z_f32(p, reinterpret_cast<float*>(q.own), nx * ny, true));
    Timed t(p, ST_SORT);
    for (int c = 0; c < q.py; ++c)
        PM_TRY_S(pencil_copy3(p, q.own + q.kb(c), ny * H, H, dst[c], ny * q.hc(c), q.hc(c), q.nx, q.ny, q.hc(c)));
    return PM_OK;
}

int pm_pencil_forward_f32(pm_pencil* pen) {
    PM_TRY_S(pencil_ok(pen));
    Pencil& q = pen->q;
    std::vector<float2*> dst(q.py);
    for (int c = 0; c < q.py; ++c) dst[c] = q.send + q.yoff(c);
    return pencil_forward_to(q, dst);
}

static int log2i(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

// The y passes read the blocks a transpose delivered and write the blocks
// the next one sends, through line maps (no staging copies):
//   y group blocks [member s][nx][ny][hc]: y = s ny + yl
//   x group blocks [member d][nx][yc][hc]: ky = d yc + kyl
// (plane = x, columns = the rank's hc kz planes; offsets below nx ng hc < 2^31).
static LineMap ymap(const Pencil& q, long long hc) {
    return LineMap{(long long)q.ny * hc, (int)((long long)q.nx * q.ny * hc), (int)hc, log2i(q.ny), q.ny - 1};
}
static LineMap kymap(const Pencil& q, long long hc) {
    return LineMap{(long long)q.yc * hc, (int)((long long)q.nx * q.yc * hc), (int)hc, log2i(q.yc), q.yc - 1};
}

int pm_pencil_yfwd_f32(pm_pencil* pen) {
    PM_TRY_S(pencil_ok(pen));
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    return pencil_lines_f32(q.plan->p, reinterpret_cast<const float*>(q.recv), reinterpret_cast<float*>(q.send),
                            ymap(q, hc), kymap(q, hc), q.nx, (int)hc, -1, ST_FFT_Y_FWD);
}

int pm_pencil_xgreen_f32(pm_pencil* pen, double c_poisson) {
    PM_TRY_S(pencil_ok(pen));
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    // the received blocks [src][nx][yc][hc] are the x lines [kx][kyl][kz]
    // (element stride yc hc), written to the same layout of send
    const LineMap m{hc, 0, (int)(q.yc * hc), 30, (1 << 30) - 1};
    return pencil_xgreen_f32(q.plan->p, reinterpret_cast<const float*>(q.recv), reinterpret_cast<float*>(q.send), m,
                             q.yc, (int)hc, c_poisson, q.rx * q.yc, q.kb(q.ry));
}

int pm_pencil_yinv_f32(pm_pencil* pen) {
    PM_TRY_S(pencil_ok(pen));
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    return pencil_lines_f32(q.plan->p, reinterpret_cast<const float*>(q.recv), reinterpret_cast<float*>(q.send),
                            kymap(q, hc), ymap(q, hc), q.nx, (int)hc, +1, ST_FFT_Y_INV);
}

// the blocks [src kz chunk][nx][ny][hc(src)] of `in` into the own rows, z
// C2R, the potential into the halo buffer's own rows
static int pencil_backward_from(Pencil& q, const float2* in) {
    const Plan& p = q.plan->p;
    const long long H = q.h, nx = q.nx, ny = q.ny;
    {
        Timed t(p, ST_SORT);
        for (int s = 0; s < q.py; ++s)
            PM_TRY_S(pencil_copy3(p, in + q.yoff(s), ny * q.hc(s), q.hc(s), q.own + q.kb(s), ny * H, H, q.nx, q.ny,
                                  q.hc(s)));
    }
    PM_TRY_S(pencil_z_f32(p, reinterpret_cast<float*>(q.own), nx * ny, false));
    Timed t(p, ST_SORT);
    return pencil_copy3(p, q.own, ny * H, H, q.halo_c() + q.hrow(2, 2), (ny + 5) * H, H, q.nx, q.ny, q.h);
}

int pm_pencil_backward_f32(pm_pencil* pen) {
    PM_TRY_S(pencil_ok(pen));
    return pencil_backward_from(pen->q, pen->q.recv);
}

// Transposes by peer stores: each pass writes its output blocks straight
// into the buffers of the group members that own them (peer device
// pointers in member order), at the block this rank's all-to-all would have
// filled; `in` is this rank's buffer the previous phase filled.
static int pencil_peers(const Pencil& q, void* const* peers, int npeers, int want, const long long* block,
                        long long ps, int s0, int n, PeerMap& po) {
    if (!peers || npeers != want) return fail(PM_ERR_ARG, "one peer buffer per group member expected");
    if (npeers > kMaxPeers) return fail(PM_ERR_SIZE, "at most 16 ranks per group for the peer-store transposes");
    for (int d = 0; d < npeers; ++d) {
        if (!peers[d]) return fail(PM_ERR_ARG, "NULL peer buffer");
        po.base[d] = static_cast<float2*>(peers[d]) + block[d];
    }
    po.ps = ps;
    po.s0 = s0;
    po.sl = log2i(n);
    po.mask = n - 1;
    (void)q;
    return PM_OK;
}

int pm_pencil_forward_peers_f32(pm_pencil* pen, void* const* peer_a, int npeers) {
    PM_TRY_S(pencil_ok(pen));
    Pencil& q = pen->q;
    if (!peer_a || npeers != q.py) return fail(PM_ERR_ARG, "one peer buffer per y-group member expected");
    for (int c = 0; c < q.py; ++c)
        if (!peer_a[c]) return fail(PM_ERR_ARG, "NULL peer buffer");
    // chunk c to member c, its block ry (blocks of nx ny hc(c))
    std::vector<float2*> dst(q.py);
    for (int c = 0; c < q.py; ++c) dst[c] = static_cast<float2*>(peer_a[c]) + (long long)q.ry * q.nx * q.ny * q.hc(c);
    return pencil_forward_to(q, dst);
}

int pm_pencil_yfwd_peers_f32(pm_pencil* pen, const void* in, void* const* peer_b, int npeers) {
    PM_TRY_S(pencil_ok(pen));
    if (!in) return fail(PM_ERR_ARG, "in is NULL");
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    // ky chunk d to x-group member d, its block rx ([nx][yc][hc])
    std::vector<long long> block(q.px, (long long)q.rx * q.nx * q.yc * hc);
    PeerMap po;
    PM_TRY_S(pencil_peers(q, peer_b, npeers, q.px, block.data(), q.yc * hc, (int)hc, q.yc, po));
    return pencil_lines_peers_f32(q.plan->p, static_cast<const float*>(in), ymap(q, hc), po, q.nx, (int)hc, -1,
                                  ST_FFT_Y_FWD);
}

int pm_pencil_xgreen_peers_f32(pm_pencil* pen, const void* in, double c_poisson, void* const* peer_a, int npeers) {
    PM_TRY_S(pencil_ok(pen));
    if (!in) return fail(PM_ERR_ARG, "in is NULL");
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    // element kx to x-group member kx / nx, its block rx, at (kx mod nx) yc hc
    std::vector<long long> block(q.px, (long long)q.rx * q.nx * q.yc * hc);
    PeerMap po;
    PM_TRY_S(pencil_peers(q, peer_a, npeers, q.px, block.data(), hc, (int)(q.yc * hc), q.nx, po));
    const LineMap m{hc, 0, (int)(q.yc * hc), 30, (1 << 30) - 1};
    return pencil_xgreen_peers_f32(q.plan->p, static_cast<const float*>(in), m, po, q.yc, (int)hc, c_poisson,
                                   q.rx * q.yc, q.kb(q.ry));
}

int pm_pencil_yinv_peers_f32(pm_pencil* pen, const void* in, void* const* peer_b, int npeers) {
    PM_TRY_S(pencil_ok(pen));
    if (!in) return fail(PM_ERR_ARG, "in is NULL");
    Pencil& q = pen->q;
    const long long hc = q.hc(q.ry);
    // y block d to y-group member d, at its kz chunk ry (complex offset nx ny kb(ry))
    std::vector<long long> block(q.py, q.yoff(q.ry));
    PeerMap po;
    PM_TRY_S(pencil_peers(q, peer_b, npeers, q.py, block.data(), q.ny * hc, (int)hc, q.ny, po));
    return pencil_lines_peers_f32(q.plan->p, static_cast<const float*>(in), kymap(q, hc), po, q.nx, (int)hc, +1,
                                  ST_FFT_Y_INV);
}

int pm_pencil_backward_from_f32(pm_pencil* pen, const void* in) {
    PM_TRY_S(pencil_ok(pen));
    if (!in) return fail(PM_ERR_ARG, "in is NULL");
    return pencil_backward_from(pen->q, static_cast<const float2*>(in));
}

int pm_pencil_kick_drift_f32(pm_pencil* pen, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                             float* vz, int64_t np, double c_kick, double dt) {
    PM_TRY_S(pencil_ok(pen));
    if (np < 0) return fail(PM_ERR_ARG, "negative particle count");
    if (np > 0 && (!cell || !ox || !oy || !oz || !vx || !vy || !vz)) return fail(PM_ERR_ARG, "NULL particle array");
    Pencil& q = pen->q;
    return pencil_kick_drift_f32(q.plan->p, q.x0, q.y0, q.nx, q.ny, q.halo, cell, ox, oy, oz, vx, vy, vz, np, c_kick,
                                 dt);
}

int pm_pencil_migrate_sort(pm_pencil* pen, const uint32_t* cell, int64_t np, int64_t* counts) {
    PM_TRY_S(pencil_ok(pen));
    if (np < 0 || !counts || (np > 0 && !cell)) return fail(PM_ERR_ARG, "bad migration arguments");
    if (np > (int64_t)0xffffffffll) return fail(PM_ERR_SIZE, "a pencil holds at most 2^32 - 1 particles");
    Pencil& q = pen->q;
    return pencil_rank_sort(q.plan->p, q.px, q.py, q.nx, q.ny, cell, np, counts);
}

int pm_pencil_migrate_pack(pm_pencil* pen, void* const* arrays, int narrays, int64_t np, uint32_t* packed) {
    PM_TRY_S(pencil_ok(pen));
    if (!arrays || narrays < 1 || narrays > 8 || np < 0 || (np > 0 && !packed))
        return fail(PM_ERR_ARG, "bad pack arguments");
    Words w{};
    for (int a = 0; a < narrays; ++a) {
        w.a[a] = static_cast<uint32_t*>(arrays[a]);
        if (np > 0 && !w.a[a]) return fail(PM_ERR_ARG, "NULL particle array");
    }
    const Plan& p = pen->q.plan->p;
    if (np > p.tiles.np_cap) return fail(PM_ERR_STATE, "pm_pencil_migrate_sort must precede the pack");
    if (np == 0) return PM_OK;
    {
        Timed t(p, ST_SORT);
        k_pack_words<<<grid_for(p, np, 256, 4), 256, 0, p.stream>>>(p.tiles.perm, np, w, narrays, packed);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pm_pencil_migrate_unpack(pm_pencil* pen, const uint32_t* packed, int64_t n, void* const* arrays, int narrays,
                             int64_t at) {
    PM_TRY_S(pencil_ok(pen));
    if (!arrays || narrays < 1 || narrays > 8 || n < 0 || at < 0 || (n > 0 && !packed))
        return fail(PM_ERR_ARG, "bad unpack arguments");
    Words w{};
    for (int a = 0; a < narrays; ++a) {
        w.a[a] = static_cast<uint32_t*>(arrays[a]);
        if (n > 0 && !w.a[a]) return fail(PM_ERR_ARG, "NULL particle array");
    }
    if (n == 0) return PM_OK;
    const Plan& p = pen->q.plan->p;
    {
        Timed t(p, ST_SORT);
        k_unpack_words<<<grid_for(p, n, 256, 4), 256, 0, p.stream>>>(packed, n, w, narrays, at);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

int pm_pencil_check(pm_pencil* pen) {
    if (!pen || !pen->q.plan) return fail(PM_ERR_ARG, "pencil is NULL");
    return pm_plan_check(pen->q.plan);
}

}  // extern "C"
