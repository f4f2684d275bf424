// Tile-binned CIC deposit for the FP32 split-position path, and the spatial
// particle sort that keeps the particle arrays in tile order.
//
// The reference deposits into one private mesh per OpenMP thread and sums
// them (src/utils/utils.cpp:70-113), then folds the +1 ghost planes into
// their periodic images (src/decomp/slab/reorder_slab.cpp:43-68).  Here each
// cell is written exactly once by the block that owns its tile:
//
//   1. bucket every particle by (tile of its base cell, face class), where a
//      tile is TS^3 cells and the class has one bit per axis set when the base
//      cell lies on the tile's upper face (its +1 corner leaves the tile);
//   2. one block per tile accumulates, in shared memory, the in-tile corners
//      of its own particles and of the face particles of its seven lower
//      neighbours (whose +1 corners land in this tile), then stores the tile
//      with plain coalesced stores (background -1 added, row padding zeroed).
//
// No global atomics touch the mesh and no separate initialisation pass is
// needed.  Counting uses warp-aggregated atomics (__match_any_sync) on the
// bucket counters; the exclusive scan is a three-kernel block scan.
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <vector>

#include "fft_engine.cuh"

namespace pmb {

namespace {

constexpr int kScanThreads = 1024, kScanItems = 2;  // 2048 entries per scan block

__device__ __forceinline__ void unpack(uint32_t c, int& i, int& j, int& k) {
    i = (int)(c >> 20);
    j = (int)((c >> 10) & 1023u);
    k = (int)(c & 1023u);
}

// Bucket of a particle: ((tx * nt + ty) * nt + tz) * 8 + class.  Cell
// indices are wrapped by the mesh size, so a cell >= ng (invalid input)
// lands on its periodic image rather than outside the bucket arrays.
__device__ __forceinline__ uint32_t bucket_of(uint32_t c, int ts_log, int nt) {
    int i, j, k;
    unpack(c, i, j, k);
    const int n = nt << ts_log;
    if (i >= n) i %= n;
    if (j >= n) j %= n;
    if (k >= n) k %= n;
    const int m = (1 << ts_log) - 1;
    const uint32_t tile = ((uint32_t)(i >> ts_log) * nt + (uint32_t)(j >> ts_log)) * nt + (uint32_t)(k >> ts_log);
    const uint32_t cls = ((i & m) == m ? 1u : 0u) | ((j & m) == m ? 2u : 0u) | ((k & m) == m ? 4u : 0u);
    return tile * 8u + cls;
}

// Bucket of a particle for the column tiles of the fused deposit + z FFT:
// CT x CT cells in (x, y) and the whole z extent; class bits x-face (1),
// y-face (2).  ts_log = log2 CT, nt = tiles per axis.  zcb > 0 splits every
// (tile, class) bucket into 2^zcb z chunks, z chunk fastest, so that the
// classes of a tile still form one contiguous run of buckets.
__device__ __forceinline__ uint32_t column_bucket_of(uint32_t c, int ts_log, int nt, int zcb = 0) {
    int i, j, k;
    unpack(c, i, j, k);
    const int n = nt << ts_log;
    if (i >= n) i %= n;
    if (j >= n) j %= n;
    const int m = (1 << ts_log) - 1;
    const uint32_t tile = (uint32_t)(i >> ts_log) * nt + (uint32_t)(j >> ts_log);
    const uint32_t b = tile * 4u + ((i & m) == m ? 1u : 0u) + ((j & m) == m ? 2u : 0u);
    if (zcb == 0) return b;
    if (k >= n) k %= n;
    const int zsh = __ffs(n) - 1 - zcb;  // log2 of the chunk length
    return (b << zcb) + (uint32_t)(k >> zsh);
}

// Bucket of a particle for the column tiles of one x-slab (planes
// [x0, x0 + nxl) of the mesh): the column key of the slab-local x plane.  A
// cell outside the slab (which the slab migration never leaves behind) is
// clamped into it so that every bucket index stays in range.
__device__ __forceinline__ uint32_t slab_column_bucket_of(uint32_t c, int nt, int x0, int nxl) {
    int i, j, k;
    unpack(c, i, j, k);
    const int n = nt << 2;
    if (j >= n) j %= n;
    int li = i - x0;
    if (li < 0 || li >= nxl) {
        li = ((i % n) - x0 + n) % n;
        if (li >= nxl) li = nxl - 1;
    }
    return ((uint32_t)(li >> 2) * nt + (uint32_t)(j >> 2)) * 4u + ((li & 3) == 3 ? 1u : 0u) + ((j & 3) == 3 ? 2u : 0u);
}

// Owner of a particle in an x-slab decomposition: (i mod n) >> log2(nx).
__device__ __forceinline__ uint32_t slab_rank_of(uint32_t c, int nx_log, int n) {
    int i = (int)(c >> 20);
    if (i >= n) i %= n;
    return (uint32_t)(i >> nx_log);
}

// Owner of a particle in a pencil decomposition (Px x Py ranks, rank =
// px * Py + py): ((i mod n) >> log2 nx) << log2 Py | ((j mod n) >> log2 ny);
// yp packs log2 ny (low byte) and log2 Py (next byte).
__device__ __forceinline__ uint32_t pencil_rank_of(uint32_t c, int nx_log, int n, int yp) {
    int i = (int)(c >> 20), j = (int)((c >> 10) & 1023u);
    if (i >= n) i %= n;
    if (j >= n) j %= n;
    return ((uint32_t)(i >> nx_log) << ((yp >> 8) & 255)) | (uint32_t)(j >> (yp & 255));
}

enum : int { KEY_TILE3 = 0, KEY_MORTON = 1, KEY_COLUMN = 2, KEY_SLABCOL = 3, KEY_RANK = 4, KEY_PENCIL = 5 };

// Morton (Z-order) index of a particle's tile, for the spatial sort.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // 10 bits -> every third bit
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__device__ __forceinline__ uint32_t morton_tile(uint32_t c, int ts_log, int nt) {
    int i, j, k;
    unpack(c, i, j, k);
    const int n = nt << ts_log;
    if (i >= n) i %= n;
    if (j >= n) j %= n;
    if (k >= n) k %= n;
    return (spread3((uint32_t)(i >> ts_log)) << 2) | (spread3((uint32_t)(j >> ts_log)) << 1) |
           spread3((uint32_t)(k >> ts_log));
}

// count[key(p)] += 1, aggregated over the lanes of a warp that share a key.
// Batches: with pbeg != null, grid row blockIdx.y handles the particles
// [pbeg[b], pend[b]) of box b, whose buckets start at b * nb_box.
constexpr int kBinU = 4;  // chunks of 32 particles per warp and round in the binning kernels

// Bucket key of particle p (0xffffffff past the end; no bucket has that key).
// KEY_COLUMN reads the z-chunk bits from xa; KEY_SLABCOL reads (x0, nxl)
// from (ts_log, xa), nt the column tiles per axis; KEY_RANK reads log2 of
// the slab width from ts_log and the mesh size from nt.
template <int KEY>
__device__ __forceinline__ uint32_t bin_key(const uint32_t* __restrict__ cell, long long p, long long hi, uint32_t kb,
                                            int ts_log, int nt, int xa = 0) {
    if (p >= hi) return 0xffffffffu;
    const uint32_t c = __ldg(cell + p);
    if (KEY == KEY_SLABCOL) return kb + slab_column_bucket_of(c, nt, ts_log, xa);
    if (KEY == KEY_RANK) return kb + slab_rank_of(c, ts_log, nt);
    if (KEY == KEY_PENCIL) return kb + pencil_rank_of(c, ts_log, nt, xa);
    return kb + (KEY == KEY_MORTON ? morton_tile(c, ts_log, nt)
                                   : (KEY == KEY_COLUMN ? column_bucket_of(c, ts_log, nt, xa) : bucket_of(c, ts_log, nt)));
}

template <int KEY>
__global__ void k_bucket_count(const uint32_t* __restrict__ cell, long long np, int ts_log, int nt,
                               uint32_t* __restrict__ count, const long long* __restrict__ pbeg = nullptr,
                               const long long* __restrict__ pend = nullptr, long long nb_box = 0, int xa = 0) {
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long lo = pbeg ? pbeg[blockIdx.y] : 0, hi = pbeg ? pend[blockIdx.y] : np;
    const uint32_t kb = pbeg ? (uint32_t)(blockIdx.y * nb_box) : 0u;
    // kBinU chunks of 32 particles per warp and round, their loads in flight together
    for (long long base = lo + warp * 32 * kBinU; base < hi; base += nwarps * 32 * kBinU) {
        uint32_t key[kBinU];
#pragma unroll
        for (int u = 0; u < kBinU; ++u) key[u] = bin_key<KEY>(cell, base + u * 32 + lane, hi, kb, ts_log, nt, xa);
#pragma unroll
        for (int u = 0; u < kBinU; ++u) {
            const unsigned peers = __match_any_sync(0xffffffffu, key[u]);
            if (key[u] != 0xffffffffu && lane == __ffs(peers) - 1) atomicAdd(count + key[u], (uint32_t)__popc(peers));
        }
    }
}

// perm[cursor[key(p)]++] = p, aggregated per warp.
template <int KEY>
__global__ void k_bucket_scatter(const uint32_t* __restrict__ cell, long long np, int ts_log, int nt,
                                 uint32_t* __restrict__ cursor, uint32_t* __restrict__ perm,
                                 const long long* __restrict__ pbeg = nullptr,
                                 const long long* __restrict__ pend = nullptr, long long nb_box = 0, int xa = 0) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long lo = pbeg ? pbeg[blockIdx.y] : 0, hi = pbeg ? pend[blockIdx.y] : np;
    const uint32_t kb = pbeg ? (uint32_t)(blockIdx.y * nb_box) : 0u;
    // kBinU chunks per round: loads, then all cursor atomics, then the stores,
    // so the round trips of the chunks overlap
    for (long long base = lo + warp * 32 * kBinU; base < hi; base += nwarps * 32 * kBinU) {
        uint32_t key[kBinU], at[kBinU];
        unsigned peers[kBinU];
#pragma unroll
        for (int u = 0; u < kBinU; ++u) key[u] = bin_key<KEY>(cell, base + u * 32 + lane, hi, kb, ts_log, nt, xa);
#pragma unroll
        for (int u = 0; u < kBinU; ++u) {
            peers[u] = __match_any_sync(0xffffffffu, key[u]);
            at[u] = 0;
            if (key[u] != 0xffffffffu && lane == __ffs(peers[u]) - 1)
                at[u] = atomicAdd(cursor + key[u], (uint32_t)__popc(peers[u]));
        }
#pragma unroll
        for (int u = 0; u < kBinU; ++u) {
            const uint32_t a = __shfl_sync(0xffffffffu, at[u], __ffs(peers[u]) - 1);
            if (key[u] != 0xffffffffu) perm[a + __popc(peers[u] & lt)] = (uint32_t)(base + u * 32 + lane);
        }
    }
}

// Exclusive scan of count[0..nb) into off[0..nb] (off[nb] = total) and
// cursor[0..nb), in three steps: per-block scan, scan of block sums, add.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;  // inclusive prefix of warp sums
    }
    __syncthreads();
    total = sh[(blockDim.x >> 5) - 1];
    const uint32_t r = x - v + (w > 0 ? sh[w - 1] : 0u);
    __syncthreads();
    return r;
}

__global__ void k_scan_local(const uint32_t* __restrict__ count, long long nb, uint32_t* __restrict__ off,
                             uint32_t* __restrict__ bsum) {
    __shared__ uint32_t sh[32];
    const long long i0 = (long long)blockIdx.x * kScanThreads * kScanItems + (long long)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        v[q] = i0 + q < nb ? count[i0 + q] : 0u;
        s += v[q];
    }
    uint32_t total;
    uint32_t e = block_excl_scan(s, sh, total);
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        if (i0 + q < nb) off[i0 + q] = e;
        e += v[q];
    }
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* __restrict__ bsum, int nblocks, uint32_t* __restrict__ total_out) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (int b0 = 0; b0 < nblocks; b0 += kScanThreads) {
        const int b = b0 + threadIdx.x;
        const uint32_t v = b < nblocks ? bsum[b] : 0u;
        uint32_t tot;
        const uint32_t e = block_excl_scan(v, sh, tot);
        if (b < nblocks) bsum[b] = e + carry;
        carry += tot;
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(uint32_t* __restrict__ off, uint32_t* __restrict__ cursor, long long nb,
                           const uint32_t* __restrict__ bsum) {
    const long long i0 = (long long)blockIdx.x * kScanThreads * kScanItems + (long long)threadIdx.x * kScanItems;
    const uint32_t add = bsum[blockIdx.x];
#pragma unroll
    for (int q = 0; q < kScanItems; ++q)
        if (i0 + q < nb) {
            const uint32_t o = off[i0 + q] + add;
            off[i0 + q] = o;
            cursor[i0 + q] = o;
        }
}

// One block per tile: accumulate, store.  Source tiles are the tile itself
// (all classes) and its 7 lower neighbours, periodic, restricted to the
// classes whose bits cover the neighbour offset q.  Those classes form the
// 14 fixed runs [c0, c1) below (q = 0: all 8 classes; q = x: 1, 3, 5, 7; ...).
constexpr int kRuns = 14;
__constant__ int kRunQ[kRuns] = {0, 1, 1, 1, 1, 2, 2, 3, 3, 4, 5, 5, 6, 7};
__constant__ int kRunC0[kRuns] = {0, 1, 3, 5, 7, 2, 6, 3, 7, 4, 5, 7, 6, 7};
__constant__ int kRunC1[kRuns] = {8, 2, 4, 6, 8, 4, 8, 4, 8, 8, 6, 8, 8, 8};
template <int TS>
__global__ void __launch_bounds__(256) k_tile_deposit(const uint32_t* __restrict__ cell, const float* __restrict__ ox,
                                                      const float* __restrict__ oy, const float* __restrict__ oz,
                                                      const uint32_t* __restrict__ perm,
                                                      const uint32_t* __restrict__ off, float mass, float background,
                                                      float* __restrict__ mesh, int n, int nt,
                                                      long long mesh_stride = 0,
                                                      const float* __restrict__ box_mass = nullptr) {
    __shared__ __align__(16) float acc[TS * TS * TS];
    __shared__ uint32_t rbeg[kRuns], rpre[kRuns + 1];
    // a batch of boxes: blockIdx.x = box * nt^3 + tile, buckets from box * nt^3 * 8
    const int tpb = nt * nt * nt, box = blockIdx.x / tpb, tile = blockIdx.x % tpb;
    const int tx = tile / (nt * nt), ty = (tile / nt) % nt, tz = tile % nt;
    mesh += box * mesh_stride;
    if (box_mass) mass = box_mass[box];
    off += (size_t)box * tpb * 8;
    for (int c = threadIdx.x; c < TS * TS * TS / 4; c += blockDim.x)
        reinterpret_cast<float4*>(acc)[c] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (threadIdx.x < kRuns) {  // one bucket run per thread, loaded in parallel
        const int q = kRunQ[threadIdx.x];
        const int sx = (tx - (q & 1) + nt) % nt, sy = (ty - ((q >> 1) & 1) + nt) % nt;
        const int sz = (tz - ((q >> 2) & 1) + nt) % nt;
        const uint32_t b = (uint32_t)((sx * nt + sy) * nt + sz) * 8u;
        const uint32_t beg = __ldg(off + b + kRunC0[threadIdx.x]);
        rbeg[threadIdx.x] = beg;
        rpre[threadIdx.x + 1] = __ldg(off + b + kRunC1[threadIdx.x]) - beg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        rpre[0] = 0;
        for (int r = 0; r < kRuns; ++r) rpre[r + 1] += rpre[r];
    }
    __syncthreads();
    const uint32_t total = rpre[kRuns];
    for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
        int r = 0;
        while (t >= rpre[r + 1]) ++r;
        const uint32_t p = __ldg(perm + rbeg[r] + (t - rpre[r]));
        const int q = kRunQ[r];
        int i, j, k;
        unpack(__ldg(cell + p), i, j, k);  // (only the low ts_log bits are used below)
        // base cell in this tile's frame: local coordinate, minus TS for a
        // source tile one step below (the particle sits on its upper face)
        const int li = (i & (TS - 1)) - ((q & 1) ? TS : 0);
        const int lj = (j & (TS - 1)) - ((q & 2) ? TS : 0);
        const int lk = (k & (TS - 1)) - ((q & 4) ? TS : 0);
        const float fx = __ldg(ox + p), fy = __ldg(oy + p), fz = __ldg(oz + p);
        const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {mass * (1.0f - fz), mass * fz};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const int ci = li + a;
            if (ci < 0 || ci >= TS) continue;
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const int cj = lj + b;
                if (cj < 0 || cj >= TS) continue;
                const float wab = wx[a] * wy[b];
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int ck = lk + c;
                    if (ck < 0 || ck >= TS) continue;
                    atomicAdd(&acc[(ci * TS + cj) * TS + ck], wab * wz[c]);
                }
            }
        }
    }
    __syncthreads();
    // store as float2 pairs (mesh rows are 8-byte aligned: n + 2 is even);
    // consecutive threads take consecutive pairs of a row
    const long long pz = n + 2;
    constexpr int PAIRS = TS / 2;
    for (int c = threadIdx.x; c < TS * TS * PAIRS; c += blockDim.x) {
        const int r = c / PAIRS, ck = 2 * (c % PAIRS);  // r = ci * TS + cj
        const long long row = (long long)(tx * TS + r / TS) * n + (ty * TS + r % TS);
        float2* dst = reinterpret_cast<float2*>(mesh + row * pz + tz * TS + ck);
        const float2 v = reinterpret_cast<const float2*>(acc)[c];
        *dst = make_float2(background + v.x, background + v.y);
        if (tz == nt - 1 && ck == TS - 2) *reinterpret_cast<float2*>(mesh + row * pz + n) = make_float2(0.f, 0.f);
    }
}

// Fused deposit + z R2C.  One block per column tile of CT x CT (x, y) cells
// and the whole z extent (16 rows of N reals): the in-tile CIC corners of the
// tile's own particles and of the x / y face particles of its three lower
// neighbours are accumulated straight into the padded complex layout of the
// z FFT, then each row (minus the -1 background) is transformed in shared
// memory and written as its N/2+1 spectrum entries.  The density mesh itself
// is never stored: one write of the mesh instead of a write and a read.
constexpr int kCT = 4, kCTRows = kCT * kCT;
constexpr int kColRuns = 5;  // (q, class range): own [0,4); x-1 {1},{3}; y-1 [2,4); x-1,y-1 {3}
__constant__ int kColQ[kColRuns] = {0, 1, 1, 2, 3};
__constant__ int kColC0[kColRuns] = {0, 1, 3, 2, 3};
__constant__ int kColC1[kColRuns] = {4, 2, 4, 4, 4};

template <int N> constexpr int zcol_threads() { return kCTRows * (N / 2) / Radix<N / 2>::R2; }

// The CIC corners of one particle that land in this block's 4 x 4 columns.
// Q: the tile it is binned in, 0 this one, bit 0 the x - 1 tile (then
// i & 3 == 3 and only the a = 1 corners land here, in column 0), bit 1 the
// y - 1 tile (likewise in y).  Two z cells per corner, FP32 shared atomics
// into the padded complex rows (real index k at 2 zpad(k / 2) + k % 2).
template <int N, int R1, int RS, int Q>
__device__ __forceinline__ void zcol_corners(uint32_t c, float fx, float fy, float fz, float mass, float* Sf) {
    int i, j, k;
    unpack(c, i, j, k);
    if (k >= N) k %= N;
    const int k1 = (k + 1) & (N - 1);
    const int z0 = 2 * zpad<R1>(k >> 1) + (k & 1), z1 = 2 * zpad<R1>(k1 >> 1) + (k1 & 1);
    const float wz0 = mass * (1.0f - fz), wz1 = mass * fz;
    auto put = [&](int ci, int cj, float w) {
        float* row = Sf + (ci * kCT + cj) * (2 * RS);
        atomicAdd(row + z0, w * wz0);
        atomicAdd(row + z1, w * wz1);
    };
    const int li = i & (kCT - 1), lj = j & (kCT - 1);
    if (Q == 0) {
        put(li, lj, (1.0f - fx) * (1.0f - fy));
        if (li < kCT - 1) put(li + 1, lj, fx * (1.0f - fy));
        if (lj < kCT - 1) put(li, lj + 1, (1.0f - fx) * fy);
        if (li < kCT - 1 && lj < kCT - 1) put(li + 1, lj + 1, fx * fy);
    } else if (Q == 1) {
        put(0, lj, fx * (1.0f - fy));
        if (lj < kCT - 1) put(0, lj + 1, fx * fy);
    } else if (Q == 2) {
        put(li, 0, (1.0f - fx) * fy);
        if (li < kCT - 1) put(li + 1, 0, fx * fy);
    } else {
        put(0, 0, fx * fy);
    }
}

// Three blocks per SM (80 registers; 3 x 67.6 KB of rows at N = 1024): the
// particle phase of one block overlaps the FFT and store phases of another.
// SLAB: the tile rows of one x-slab (blockIdx.x = tx * nt + ty, tx < nx/4 + 1):
// no periodic x neighbour (tile row 0 takes no x - 1 halo; the previous
// slab's face particles arrive through its ghost plane), and the tile rows
// from ntx_own on -- the ghost row, whose plane 0 holds the +1 corners of the
// slab's last plane -- carry no -1 background.
template <int N, bool SLAB = false>
__global__ void __launch_bounds__(zcol_threads<N>(), 3)
k_deposit_zr2c(const uint32_t* __restrict__ cell, const float* __restrict__ ox, const float* __restrict__ oy,
               const float* __restrict__ oz, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ off,
               float mass, float* __restrict__ mesh, const float2* __restrict__ tw, int nt, long long nb_box = 0,
               long long mesh_stride = 0, const float* __restrict__ box_mass = nullptr, int ntx_own = 0,
               int zcb = 0) {
    // a batch of boxes: box blockIdx.y has its own buckets, mesh and mass
    if (box_mass) mass = __ldg(box_mass + blockIdx.y);
    off += blockIdx.y * nb_box;
    mesh += blockIdx.y * mesh_stride;
    constexpr int M = N / 2, R1 = Radix<M>::R1, R2 = Radix<M>::R2, NT = M / R2, RS = z_row_stride<N>();
    constexpr int NTH = zcol_threads<N>();
    using I = ZIdx<R1, R2>;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2* S = reinterpret_cast<float2*>(smraw);
    float* Sf = reinterpret_cast<float*>(smraw);
    __shared__ uint32_t rbeg[kColRuns], rpre[kColRuns + 1];
    const int tile = blockIdx.x, tx = tile / nt, ty = tile % nt;
    for (int c = threadIdx.x; c < kCTRows * RS; c += NTH) S[c] = make_float2(0.f, 0.f);
    if (threadIdx.x < kColRuns) {
        const int q = kColQ[threadIdx.x];
        const int sx = SLAB ? tx - (q & 1) : (tx - (q & 1) + nt) % nt, sy = (ty - ((q >> 1) & 1) + nt) % nt;
        if (SLAB && sx < 0) {  // the slab's first tile row: no x - 1 neighbour here
            rbeg[threadIdx.x] = 0;
            rpre[threadIdx.x + 1] = 0;
        } else {
            // (with z chunks, a class range of the tile spans its chunks)
            const uint32_t b = (uint32_t)(sx * nt + sy) * 4u;
            const uint32_t beg = __ldg(off + ((b + kColC0[threadIdx.x]) << zcb));
            rbeg[threadIdx.x] = beg;
            rpre[threadIdx.x + 1] = __ldg(off + ((b + kColC1[threadIdx.x]) << zcb)) - beg;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        rpre[0] = 0;
        for (int r = 0; r < kColRuns; ++r) rpre[r + 1] += rpre[r];
    }
    __syncthreads();
    const uint32_t total = rpre[kColRuns];
    // run r covers t in [rpre[r], rpre[r+1]) at perm index t + rbeg[r] - rpre[r]
    // (unsigned wrap-around is exact); the boundaries stay in registers
    const uint32_t p1 = rpre[1], p2 = rpre[2], p3 = rpre[3], p4 = rpre[4];
    const uint32_t d0 = rbeg[0], d1 = rbeg[1] - p1, d2 = rbeg[2] - p2, d3 = rbeg[3] - p3, d4 = rbeg[4] - p4;
    // four particles per thread per round, their loads issued together
    constexpr int U = 4;
    for (uint32_t t0 = threadIdx.x; t0 < total; t0 += U * NTH) {
        uint32_t pidx[U];
        int qq[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t t = t0 + u * NTH;
            uint32_t d = d0;
            int q = 0;
            if (t >= p1) d = d1, q = 1;
            if (t >= p2) d = d2;  // the x - 1 tile's second class, still q = 1
            if (t >= p3) d = d3, q = 2;
            if (t >= p4) d = d4, q = 3;
            const bool ok = t < total;
            pidx[u] = ok ? __ldg(perm + (t + d)) : 0u;
            qq[u] = ok ? q : -1;
        }
        uint32_t cc[U];
        float fx[U], fy[U], fz[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (qq[u] < 0) continue;
            cc[u] = __ldg(cell + pidx[u]);
            fx[u] = __ldg(ox + pidx[u]);
            fy[u] = __ldg(oy + pidx[u]);
            fz[u] = __ldg(oz + pidx[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            // q is uniform across a warp except at run boundaries
            switch (qq[u]) {
                case 0: zcol_corners<N, R1, RS, 0>(cc[u], fx[u], fy[u], fz[u], mass, Sf); break;
                case 1: zcol_corners<N, R1, RS, 1>(cc[u], fx[u], fy[u], fz[u], mass, Sf); break;
                case 2: zcol_corners<N, R1, RS, 2>(cc[u], fx[u], fy[u], fz[u], mass, Sf); break;
                case 3: zcol_corners<N, R1, RS, 3>(cc[u], fx[u], fy[u], fz[u], mass, Sf); break;
                default: break;
            }
        }
    }
    __syncthreads();
    // z R2C of the 16 rows (the z pass of the FFT, input already in shared memory)
    const int rrow = threadIdx.x / NT, tj = threadIdx.x % NT;
    float2* R = S + rrow * RS;
    const float bg = (!SLAB || tx < ntx_own) ? 1.0f : 0.0f;  // the -1 background
    stockham_pass1<R1, R2, -1, true, float2>(
        tj, [&](int j, int r) { const float2 v = R[I::in1(j, r)]; return make_float2(v.x - bg, v.y - bg); },
        [&](int j, int k, float2 v) { R[I::out1(j, k)] = v; });
    __syncthreads();
    // pass-2 twiddles from 10 table loads per thread (3.80 vs 4.27 ms at
    // 1024^3 with 512^3 particles on B200); the outputs stay in registers and
    // the real-FFT post-processing pairs them across lanes by shuffles
    // instead of a second shared-memory round trip (3.70 vs 3.82 ms)
    float2 X[R2];
    stockham_pass2<R1, R2, -1, false, float2>(
        tj, [&](int j, int r) { return R[I::p2(j, r)]; }, [&](int, int k, float2 v) { X[k] = v; },
        pass2_twiddles<-1, (R2 >= 16), 2>(tw, tj));
    const int ci = rrow / kCT, cj = rrow % kCT;
    float2* crow = reinterpret_cast<float2*>(mesh + ((long long)(tx * kCT + ci) * N + (ty * kCT + cj)) * (N + 2));
    r2c_post<R1, R2, float2>(X, tj, true, crow, tw);
}

// out[i] = in[perm[i]] for the seven particle arrays (32-bit words).
__global__ void k_gather7(const uint32_t* __restrict__ perm, long long np, const uint32_t* const* __restrict__ src,
                          uint32_t* const* __restrict__ dst) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < np;
         i += (long long)gridDim.x * blockDim.x) {
        const uint32_t p = perm[i];
#pragma unroll
        for (int a = 0; a < 7; ++a) dst[a][i] = __ldg(src[a] + p);
    }
}

// 16^3 tiles where 16 divides the mesh, else 8^3 (the 8^3 mesh and the
// mixed-radix sizes 24, 40, 120).
int tile_log(int n) { return n % 16 == 0 ? 4 : 3; }

// Counting sort of the bucket keys into perm / off (scratch of the plan).
template <int KEY>
int bucket_sort(const Plan& p, const uint32_t* cell, int64_t np, int ts_log, int nt, long long nb, TileScratch& s,
                int xa = 0) {
    const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const unsigned g = grid_for(p, np, 256);
    {
        Timed t(p, ST_BIN, np > 0 ? 5 : 3);  // count, three scan kernels, scatter
        if (np > 0) k_bucket_count<KEY><<<g, 256, 0, p.stream>>>(cell, np, ts_log, nt, s.count, nullptr, nullptr, 0, xa);
        k_scan_local<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, (int)nscan, s.off + nb);
        k_scan_add<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        if (np > 0)
            k_bucket_scatter<KEY><<<g, 256, 0, p.stream>>>(cell, np, ts_log, nt, s.cursor, s.perm, nullptr, nullptr, 0, xa);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

}  // namespace

int tile_scratch_ensure(Plan& p, int64_t np, int nbox, long long min_nb) {
    // the permutation and the bucket offsets are 32-bit particle indices
    if (np > (int64_t)0xffffffffll) return fail(PM_ERR_SIZE, "the FP32 binning holds at most 2^32 - 1 particles");
    const int ts = 1 << tile_log(p.ng), nt = p.ng / ts;
    int nt2 = 1;  // the sort's Morton keys need nt2^3 buckets
    while (nt2 < nt) nt2 <<= 1;
    // the largest bucket layout: 3D tiles x 8 classes, Morton keys, or the
    // fused deposit's column tiles x 4 classes
    const long long col = (long long)(p.ng / 4) * (p.ng / 4) * 4;
    const long long per = std::max(std::max((long long)nt * nt * nt * 8, (long long)nt2 * nt2 * nt2), col);
    const long long nb = std::max(per * nbox, min_nb);
    TileScratch& s = p.tiles;
    if (s.nb < nb) {
        for (uint32_t** q : {&s.count, &s.off, &s.cursor, &s.bsum}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
        }
        const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
        if (cudaMalloc(&s.count, nb * 4) != cudaSuccess || cudaMalloc(&s.off, (nb + 1) * 4) != cudaSuccess ||
            cudaMalloc(&s.cursor, nb * 4) != cudaSuccess || cudaMalloc(&s.bsum, nscan * 4) != cudaSuccess) {
            cudaGetLastError();
            s.nb = 0;
            return fail(PM_ERR_NOMEM, "tile scratch allocation failed");
        }
        s.nb = nb;
        p.bytes += (size_t)(nb * 3 + 1 + nscan) * 4;
    }
    if (s.np_cap < np) {
        if (s.perm) cudaFree(s.perm);
        s.perm = nullptr;
        if (cudaMalloc(&s.perm, (size_t)np * 4) != cudaSuccess) {
            cudaGetLastError();
            s.np_cap = 0;
            return fail(PM_ERR_NOMEM, "tile scratch allocation failed");
        }
        p.bytes += (size_t)(np - s.np_cap) * 4;
        s.np_cap = np;
    }
    return PM_OK;
}

void tile_scratch_release(Plan& p) {
    TileScratch& s = p.tiles;
    for (uint32_t* q : {s.count, s.off, s.cursor, s.bsum, s.perm})
        if (q) cudaFree(q);
    s = TileScratch{};
}

int deposit_f32_tiles(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz, int64_t np,
                      float mass, float* mesh) {
    const int tl = tile_log(p.ng), ts = 1 << tl, nt = p.ng / ts;
    const long long nb = (long long)nt * nt * nt * 8;
    int rc = tile_scratch_ensure(p, np > 0 ? np : 1, 1);
    if (rc != PM_OK) return rc;
    rc = bucket_sort<KEY_TILE3>(p, cell, np, tl, nt, nb, p.tiles);
    if (rc != PM_OK) return rc;
    {
        Timed t(p, ST_DEPOSIT);
        if (ts == 16)
            k_tile_deposit<16><<<nt * nt * nt, 256, 0, p.stream>>>(cell, ox, oy, oz, p.tiles.perm, p.tiles.off, mass,
                                                                  -1.0f, mesh, p.ng, nt);
        else
            k_tile_deposit<8><<<nt * nt * nt, 256, 0, p.stream>>>(cell, ox, oy, oz, p.tiles.perm, p.tiles.off, mass,
                                                                 -1.0f, mesh, p.ng, nt);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// A batch of nbox boxes of the plan's size: box b's particles are
// [pbeg[b], pend[b]) of the shared arrays (device ranges), its mesh is
// mesh + b * mesh_elems(ng), its particle mass box_mass[b] (device).
int deposit_f32_tiles_batch(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                            const long long* pbeg, const long long* pend, int nbox, int64_t np_total,
                            const float* box_mass, float* mesh) {
    const int tl = tile_log(p.ng), ts = 1 << tl, nt = p.ng / ts;
    const long long nb_box = (long long)nt * nt * nt * 8, nb = nb_box * nbox;
    int rc = tile_scratch_ensure(p, np_total > 0 ? np_total : 1, nbox);
    if (rc != PM_OK) return rc;
    TileScratch& s = p.tiles;
    const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const long long per_box = (np_total + nbox - 1) / nbox;
    dim3 g(grid_for(p, per_box, 256, 2), nbox);
    {
        Timed t(p, ST_BIN, 5);  // count, three scan kernels, scatter
        k_bucket_count<KEY_TILE3><<<g, 256, 0, p.stream>>>(cell, np_total, tl, nt, s.count, pbeg, pend, nb_box);
        k_scan_local<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, (int)nscan, s.off + nb);
        k_scan_add<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        k_bucket_scatter<KEY_TILE3><<<g, 256, 0, p.stream>>>(cell, np_total, tl, nt, s.cursor, s.perm, pbeg, pend, nb_box);
    }
    {
        Timed t(p, ST_DEPOSIT);
        const unsigned blocks = (unsigned)(nt * nt * nt) * (unsigned)nbox;
        const long long ms = (long long)mesh_elems(p.ng);
        if (ts == 16)
            k_tile_deposit<16><<<blocks, 256, 0, p.stream>>>(cell, ox, oy, oz, s.perm, s.off, 0.0f, -1.0f, mesh,
                                                            p.ng, nt, ms, box_mass);
        else
            k_tile_deposit<8><<<blocks, 256, 0, p.stream>>>(cell, ox, oy, oz, s.perm, s.off, 0.0f, -1.0f, mesh,
                                                           p.ng, nt, ms, box_mass);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

bool zcol_supported(int ng) { return ng >= 32 && ng <= 1024 && (ng & (ng - 1)) == 0; }

template <int N> static int zcol_prepare() {
    const int smem = kCTRows * z_row_stride<N>() * (int)sizeof(float2);
    PMB_CUDA_CHECK(cudaFuncSetAttribute(k_deposit_zr2c<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    PMB_CUDA_CHECK(cudaFuncSetAttribute(k_deposit_zr2c<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return PM_OK;
}

int deposit_zr2c_prepare(const Plan& p) {
    switch (p.ng) {
        case 32: return zcol_prepare<32>();
        case 64: return zcol_prepare<64>();
        case 128: return zcol_prepare<128>();
        case 256: return zcol_prepare<256>();
        case 512: return zcol_prepare<512>();
        case 1024: return zcol_prepare<1024>();
        default: return PM_OK;
    }
}

template <int N>
static void launch_zcol(const Plan& p, unsigned blocks, const uint32_t* cell, const float* ox, const float* oy,
                        const float* oz, float mass, float* mesh, const float2* tw, int nt, int nbox = 1,
                        long long nb_box = 0, const float* box_mass = nullptr, int zcb = 0) {
    k_deposit_zr2c<N><<<dim3(blocks, nbox), zcol_threads<N>(), kCTRows * z_row_stride<N>() * sizeof(float2),
                        p.stream>>>(cell, ox, oy, oz, p.tiles.perm, p.tiles.off, mass, mesh, tw, nt, nb_box,
                                    (long long)mesh_elems(N), box_mass, 0, zcb);
}

// Deposit + z R2C in one pass over the mesh (FP32, power-of-two ng >= 32):
// mesh receives the z-transformed density contrast, ready for the y pass.
// zcb > 0 bins by (column tile, class, z chunk) for the tiled gather.
int deposit_zr2c_f32(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz, int64_t np,
                     float mass, float* mesh, int zcb) {
    const int nt = p.ng / kCT, cl = 2;  // log2 kCT
    const long long nb = ((long long)nt * nt * 4) << zcb;
    int rc = tile_scratch_ensure(p, np > 0 ? np : 1, 1, nb);
    if (rc != PM_OK) return rc;
    rc = bucket_sort<KEY_COLUMN>(p, cell, np, cl, nt, nb, p.tiles, zcb);
    if (rc != PM_OK) return rc;
    const float2* tw = static_cast<const float2*>(p.tw);
    {
        Timed t(p, ST_DEPOSIT);
        const unsigned blocks = (unsigned)(nt * nt);
        switch (p.ng) {
            case 32: launch_zcol<32>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            case 64: launch_zcol<64>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            case 128: launch_zcol<128>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            case 256: launch_zcol<256>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            case 512: launch_zcol<512>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            case 1024: launch_zcol<1024>(p, blocks, cell, ox, oy, oz, mass, mesh, tw, nt, 1, 0, nullptr, zcb); break;
            default: return fail(PM_ERR_SIZE, "fused deposit needs a power-of-two ng >= 32");
        }
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// The same for a batch of nbox boxes of one mesh size (meshes back to back,
// particles of box b in [pbeg[b], pend[b]), masses box_mass[b]).
int deposit_zr2c_f32_batch(Plan& p, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                           const long long* pbeg, const long long* pend, int nbox, int64_t np_total,
                           const float* box_mass, float* mesh) {
    const int nt = p.ng / kCT, cl = 2;  // log2 kCT
    const long long nb_box = (long long)nt * nt * 4, nb = nb_box * nbox;
    int rc = tile_scratch_ensure(p, np_total > 0 ? np_total : 1, nbox);
    if (rc != PM_OK) return rc;
    TileScratch& s = p.tiles;
    const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const long long per_box = (np_total + nbox - 1) / nbox;
    dim3 g(grid_for(p, per_box, 256, 2), nbox);
    {
        Timed t(p, ST_BIN, 5);  // count, three scan kernels, scatter
        k_bucket_count<KEY_COLUMN><<<g, 256, 0, p.stream>>>(cell, np_total, cl, nt, s.count, pbeg, pend, nb_box);
        k_scan_local<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, (int)nscan, s.off + nb);
        k_scan_add<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        k_bucket_scatter<KEY_COLUMN><<<g, 256, 0, p.stream>>>(cell, np_total, cl, nt, s.cursor, s.perm, pbeg, pend,
                                                              nb_box);
    }
    const float2* tw = static_cast<const float2*>(p.tw);
    {
        Timed t(p, ST_DEPOSIT);
        const unsigned blocks = (unsigned)(nt * nt);
        switch (p.ng) {
            case 32: launch_zcol<32>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            case 64: launch_zcol<64>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            case 128: launch_zcol<128>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            case 256: launch_zcol<256>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            case 512: launch_zcol<512>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            case 1024: launch_zcol<1024>(p, blocks, cell, ox, oy, oz, 0.f, mesh, tw, nt, nbox, nb_box, box_mass); break;
            default: return fail(PM_ERR_SIZE, "fused deposit needs a power-of-two ng >= 32");
        }
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// ------------------------------------------------------ x-slab decomposition
// Deposit of one x-slab (planes [x0, x0 + nx) of an ng^3 mesh) fused with the
// z R2C, into `mesh` = the slab's first own plane: own planes 0..nx-1 receive
// the z-transformed density contrast (background -1), planes nx..nx+3 the
// ghost tile row, whose plane nx holds the z-transformed +1 corners of the
// slab's last plane (background 0) -- the ghost plane the reference sends
// with its cube (src/decomp/slab/transpose_slab.cpp:23-27) and folds into
// the next slab (src/decomp/slab/reorder_slab.cpp:43-68).  Every particle
// must lie in the slab.
int slab_deposit_zr2c_f32(Plan& p, int x0, int nx, const uint32_t* cell, const float* ox, const float* oy,
                          const float* oz, int64_t np, float mass, float* mesh) {
    const int nt = p.ng / kCT, ntx = nx / kCT + 1;
    const long long nb = (long long)ntx * nt * 4;
    int rc = tile_scratch_ensure(p, np > 0 ? np : 1, 1, nb);
    if (rc != PM_OK) return rc;
    TileScratch& s = p.tiles;
    const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const unsigned g = grid_for(p, np, 256);
    {
        Timed t(p, ST_BIN, np > 0 ? 5 : 3);
        if (np > 0)
            k_bucket_count<KEY_SLABCOL><<<g, 256, 0, p.stream>>>(cell, np, x0, nt, s.count, nullptr, nullptr, 0, nx);
        k_scan_local<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, (int)nscan, s.off + nb);
        k_scan_add<<<(unsigned)nscan, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        if (np > 0)
            k_bucket_scatter<KEY_SLABCOL><<<g, 256, 0, p.stream>>>(cell, np, x0, nt, s.cursor, s.perm, nullptr, nullptr,
                                                                   0, nx);
    }
    const float2* tw = static_cast<const float2*>(p.tw);
    {
        Timed t(p, ST_DEPOSIT);
        const unsigned blocks = (unsigned)(ntx * nt);
        auto go = [&](auto nc) {
            constexpr int N = decltype(nc)::value;
            k_deposit_zr2c<N, true><<<blocks, zcol_threads<N>(), kCTRows * z_row_stride<N>() * sizeof(float2),
                                      p.stream>>>(cell, ox, oy, oz, s.perm, s.off, mass, mesh, tw, nt, 0, 0, nullptr,
                                                  nx / kCT);
        };
        switch (p.ng) {
            case 32: go(std::integral_constant<int, 32>{}); break;
            case 64: go(std::integral_constant<int, 64>{}); break;
            case 128: go(std::integral_constant<int, 128>{}); break;
            case 256: go(std::integral_constant<int, 256>{}); break;
            case 512: go(std::integral_constant<int, 512>{}); break;
            case 1024: go(std::integral_constant<int, 1024>{}); break;
            default: return fail(PM_ERR_SIZE, "slab deposit needs a power-of-two ng in [32, 1024]");
        }
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

// Counting sort of the particles by owning slab (x plane >> log2 nx): the
// permutation in the plan's scratch, counts[r] (host) particles per rank r.
int slab_rank_sort(Plan& p, int nranks, int nx, const uint32_t* cell, int64_t np, int64_t* counts) {
    int nx_log = 0;
    while ((1 << nx_log) < nx) ++nx_log;
    const long long nb = nranks;
    int rc = tile_scratch_ensure(p, np > 0 ? np : 1, 1, nb);
    if (rc != PM_OK) return rc;
    TileScratch& s = p.tiles;
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const unsigned g = grid_for(p, np, 256);
    {
        Timed t(p, ST_SORT, np > 0 ? 5 : 3);
        if (np > 0) k_bucket_count<KEY_RANK><<<g, 256, 0, p.stream>>>(cell, np, nx_log, p.ng, s.count);
        k_scan_local<<<1, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, 1, s.off + nb);
        k_scan_add<<<1, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        if (np > 0) k_bucket_scatter<KEY_RANK><<<g, 256, 0, p.stream>>>(cell, np, nx_log, p.ng, s.cursor, s.perm);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    std::vector<uint32_t> off(nb + 1);
    PMB_CUDA_CHECK(cudaMemcpyAsync(off.data(), s.off, (nb + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, p.stream));
    PMB_CUDA_CHECK(cudaStreamSynchronize(p.stream));
    for (long long r = 0; r < nb; ++r) counts[r] = (int64_t)off[r + 1] - (int64_t)off[r];
    return PM_OK;
}

// Counting sort of the particles by owning pencil: the permutation in the
// plan's scratch, counts[r] (host) particles per rank r = px * Py + py.
int pencil_rank_sort(Plan& p, int px, int py, int nx, int ny, const uint32_t* cell, int64_t np, int64_t* counts) {
    auto lg = [](int v) {
        int l = 0;
        while ((1 << l) < v) ++l;
        return l;
    };
    const int nx_log = lg(nx), yp = lg(ny) | (lg(py) << 8);
    const long long nb = (long long)px * py;
    int rc = tile_scratch_ensure(p, np > 0 ? np : 1, 1, nb);
    if (rc != PM_OK) return rc;
    TileScratch& s = p.tiles;
    PMB_CUDA_CHECK(cudaMemsetAsync(s.count, 0, nb * sizeof(uint32_t), p.stream));
    const unsigned g = grid_for(p, np, 256);
    {
        Timed t(p, ST_SORT, np > 0 ? 5 : 3);
        if (np > 0)
            k_bucket_count<KEY_PENCIL><<<g, 256, 0, p.stream>>>(cell, np, nx_log, p.ng, s.count, nullptr, nullptr, 0, yp);
        k_scan_local<<<1, kScanThreads, 0, p.stream>>>(s.count, nb, s.off, s.bsum);
        k_scan_sums<<<1, kScanThreads, 0, p.stream>>>(s.bsum, 1, s.off + nb);
        k_scan_add<<<1, kScanThreads, 0, p.stream>>>(s.off, s.cursor, nb, s.bsum);
        if (np > 0)
            k_bucket_scatter<KEY_PENCIL><<<g, 256, 0, p.stream>>>(cell, np, nx_log, p.ng, s.cursor, s.perm, nullptr,
                                                                  nullptr, 0, yp);
    }
    PMB_CUDA_CHECK(cudaGetLastError());
    std::vector<uint32_t> off(nb + 1);
    PMB_CUDA_CHECK(cudaMemcpyAsync(off.data(), s.off, (nb + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, p.stream));
    PMB_CUDA_CHECK(cudaStreamSynchronize(p.stream));
    for (long long r = 0; r < nb; ++r) counts[r] = (int64_t)off[r + 1] - (int64_t)off[r];
    return PM_OK;
}

int sort_f32(Plan& p, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy, float* vz, int64_t np) {
    if (np == 0) return PM_OK;
    const int tl = tile_log(p.ng), nt = p.ng >> tl;
    int nt2 = 1;  // Morton keys of nt tiles per axis lie in [0, nt2^3), nt2 the next power of two
    while (nt2 < nt) nt2 <<= 1;
    const long long nb = (long long)nt2 * nt2 * nt2;
    int rc = tile_scratch_ensure(p, np, 1);
    if (rc != PM_OK) return rc;
    rc = bucket_sort<KEY_MORTON>(p, cell, np, tl, nt, nb, p.tiles);
    if (rc != PM_OK) return rc;
    uint32_t* tmp = nullptr;
    if (cudaMallocAsync(&tmp, (size_t)np * 7 * 4, p.stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(PM_ERR_NOMEM, "sort: temporary allocation failed");
    }
    uint32_t* arrays[7] = {cell, reinterpret_cast<uint32_t*>(ox), reinterpret_cast<uint32_t*>(oy),
                           reinterpret_cast<uint32_t*>(oz), reinterpret_cast<uint32_t*>(vx),
                           reinterpret_cast<uint32_t*>(vy), reinterpret_cast<uint32_t*>(vz)};
    uint32_t* outs[7];
    for (int a = 0; a < 7; ++a) outs[a] = tmp + (size_t)a * np;
    uint32_t** dptr = nullptr;
    if (cudaMallocAsync(&dptr, 14 * sizeof(uint32_t*), p.stream) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(tmp, p.stream);
        return fail(PM_ERR_NOMEM, "sort: temporary allocation failed");
    }
    uint32_t* hptr[14];
    for (int a = 0; a < 7; ++a) {
        hptr[a] = arrays[a];
        hptr[7 + a] = outs[a];
    }
    cudaMemcpyAsync(dptr, hptr, sizeof(hptr), cudaMemcpyHostToDevice, p.stream);
    {
        Timed t(p, ST_SORT);
        k_gather7<<<grid_for(p, np, 256), 256, 0, p.stream>>>(p.tiles.perm, np, dptr, dptr + 7);
    }
    for (int a = 0; a < 7; ++a)
        cudaMemcpyAsync(arrays[a], outs[a], (size_t)np * 4, cudaMemcpyDeviceToDevice, p.stream);
    cudaFreeAsync(dptr, p.stream);
    cudaFreeAsync(tmp, p.stream);
    // the host copy of the pointer table must outlive the async copy
    PMB_CUDA_CHECK(cudaStreamSynchronize(p.stream));
    PMB_CUDA_CHECK(cudaGetLastError());
    return PM_OK;
}

}  // namespace pmb

// ------------------------------------------------ allocation-free deposit
// pm_deposit_f32_noalloc: the tile-binned FP32 deposit for callers that
// cannot allocate device memory themselves -- code running under a host
// framework whose allocator owns every device allocation, or a per-step
// path that must not allocate.  Its scratch (bucket counters, offsets,
// cursors, scan sums, permutation) is this file-scope array: every GPU that
// loads the library holds it until the process exits.
namespace pmb {
namespace {

constexpr int kNoAllocMaxNg = 256;
constexpr long long kNoAllocMaxNp = 1LL << 21;
constexpr long long kNoAllocMaxBuckets = (long long)(kNoAllocMaxNg / 16) * (kNoAllocMaxNg / 16) *
                                         (kNoAllocMaxNg / 16) * 8;
constexpr long long kNoAllocScanBlocks = (kNoAllocMaxBuckets + kScanThreads * kScanItems - 1) /
                                         (kScanThreads * kScanItems);
constexpr size_t kNoAllocWords = (size_t)(3 * kNoAllocMaxBuckets + 1 + kNoAllocScanBlocks + kNoAllocMaxNp);

__device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// The device address of g_noalloc_scratch, looked up once per device with
// that device current (a host-side use of the symbol's name is not a device
// address).
struct NoAllocDevice {
    uint32_t* scratch = nullptr;
    int num_sms = 0;
    bool ready = false;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

int noalloc_device(NoAllocDevice** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(PM_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (!d.ready) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        e = cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
        d.scratch = static_cast<uint32_t*>(ptr);
        d.ready = true;
    }
    *out = &d;
    return PM_OK;
}

}  // namespace

}  // namespace pmb

extern "C" int pm_deposit_f32_noalloc(int ng, const uint32_t* cell, const float* ox, const float* oy,
                                      const float* oz, int64_t np, float mass, float* mesh, void* stream) {
    using namespace pmb;
    if (!(ng >= 8 && ng <= kNoAllocMaxNg && (ng & (ng - 1)) == 0))
        return fail(PM_ERR_SIZE, "pm_deposit_f32_noalloc: ng must be a power of two in [8, 256]");
    if (np < 0) return fail(PM_ERR_ARG, "pm_deposit_f32_noalloc: negative particle count");
    if (np > kNoAllocMaxNp)
        return fail(PM_ERR_SIZE, "pm_deposit_f32_noalloc: at most 2097152 particles (static scratch limit)");
    if (!mesh || (np > 0 && (!cell || !ox || !oy || !oz)))
        return fail(PM_ERR_ARG, "pm_deposit_f32_noalloc: NULL array");
    NoAllocDevice* d = nullptr;
    int rc = noalloc_device(&d);
    if (rc != PM_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int tl = tile_log(ng), ts = 1 << tl, nt = ng / ts;
    const long long nb = (long long)nt * nt * nt * 8;
    const long long nscan = (nb + kScanThreads * kScanItems - 1) / (kScanThreads * kScanItems);
    uint32_t* count = d->scratch;
    uint32_t* off = count + nb;
    uint32_t* cursor = off + nb + 1;
    uint32_t* bsum = cursor + nb;
    uint32_t* perm = bsum + nscan;
    // the array keeps the previous call's contents: counters start at zero
    cudaError_t e = cudaMemsetAsync(count, 0, (size_t)nb * sizeof(uint32_t), s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync");
    long long need = (np + 255) / 256, cap = (long long)d->num_sms * 8;
    const unsigned g = (unsigned)(need < 1 ? 1 : (need < cap ? need : cap));
    if (np > 0) k_bucket_count<KEY_TILE3><<<g, 256, 0, s>>>(cell, np, tl, nt, count);
    k_scan_local<<<(unsigned)nscan, kScanThreads, 0, s>>>(count, nb, off, bsum);
    k_scan_sums<<<1, kScanThreads, 0, s>>>(bsum, (int)nscan, off + nb);
    k_scan_add<<<(unsigned)nscan, kScanThreads, 0, s>>>(off, cursor, nb, bsum);
    if (np > 0) k_bucket_scatter<KEY_TILE3><<<g, 256, 0, s>>>(cell, np, tl, nt, cursor, perm);
    if (ts == 16)
        k_tile_deposit<16><<<nt * nt * nt, 256, 0, s>>>(cell, ox, oy, oz, perm, off, mass, -1.0f, mesh, ng, nt);
    else
        k_tile_deposit<8><<<nt * nt * nt, 256, 0, s>>>(cell, ox, oy, oz, perm, off, mass, -1.0f, mesh, ng, nt);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pm_deposit_f32_noalloc launch");
    return PM_OK;
}
