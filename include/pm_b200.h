/*
 * pm_b200.h -- C ABI of the B200 particle-mesh step.
 *
 * One periodic box of ng^3 cells, particles in cell units [0, ng).  Every
 * entry point returns an int status (PM_OK = 0); pm_last_error() gives the
 * message of the calling thread's last failure.  All array arguments are
 * DEVICE pointers unless the name says host; work is enqueued on the plan's
 * stream and is asynchronous.  A plan is not thread-safe.
 *
 * Mesh layouts (row-major, z fastest):
 *   mesh      real  [ng][ng][ng+2]     the reference's FFTW in-place stride
 *                                      (src/core/main.cpp:24-28); the last two
 *                                      z entries are padding
 *   spectrum  cplx  [ng][ng][ng/2+1]   the same bytes after pm_fft_r2c*,
 *                                      kx major, kz fastest
 *   force     real  [ng][ng][ng]       one array per component
 *
 * Reference step (src/core/main.cpp:90-139) and the entry points that
 * replace its stages:
 *   init_buf + deposit_particles + reduce_private_to_shared +
 *   TransposeSlab + ReorderSlab                 -> pm_deposit_f64
 *   FFT::forward                                -> pm_fft_r2c_f64
 *   FFT::apply_green                            -> pm_green_f64
 *   FFT::backward                               -> pm_fft_c2r_f64
 *   ReorderSlabBack + TransposeSlabBack +
 *   centered_derivatives                        -> pm_gradient_f64
 *   update_particles                            -> pm_interp_kick_f64
 * On one GPU the MPI exchanges disappear: ghost planes become periodic
 * index wraps inside the kernels.
 *
 * Coefficients.  The reference hard-codes its constants
 * (include/utils/utils_inline.h:13-17).  Here they are arguments:
 *   c_poisson: phi solves  L phi = c_poisson * delta, L the 7-point
 *              Laplacian (PM_GREEN_DISCRETE, the reference) or the exact
 *              -|k|^2 (PM_GREEN_SPECTRAL); the reference value is
 *              3 Omega_0 / (2 a) with a = 0.9 (src/fft/fftw/fft.cpp:55,79).
 *   c_kick:    p += c_kick * interpolated force; the reference value is
 *              Da * function_a(a) (src/utils/utils.cpp:142).
 */
#ifndef PM_B200_H
#define PM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* status codes */
#define PM_OK 0
#define PM_ERR_ARG 1          /* null pointer, negative count, bad enum   */
#define PM_ERR_SIZE 2         /* size not supported by the library         */
#define PM_ERR_CUDA 3         /* CUDA runtime error                        */
#define PM_ERR_NOMEM 4        /* device allocation failed                  */
#define PM_ERR_RANGE 5        /* a particle position was NaN or outside
                                 [0, ng); it was wrapped (NaN -> 0) and the
                                 step completed.  Reported by pm_plan_check */
#define PM_ERR_STATE 6        /* call out of order / wrong plan precision  */

/* plan precision */
#define PM_FP64 0             /* plain FP64 path (reference parity)        */
#define PM_FP32 1             /* FP32 mesh / FFT / forces, split positions */

/* Green's function */
#define PM_GREEN_DISCRETE 0   /* inverse 7-point Laplacian (reference)     */
#define PM_GREEN_SPECTRAL 1   /* -1/|k|^2                                   */

typedef struct pm_plan pm_plan;

/* ------------------------------------------------------------ plans */

/* Creates a plan for an ng^3 mesh.  ng is a power of two in [8, 1024] or one
 * of the mixed-radix sizes 2^a 3^b 5^c 24, 40, 48, 80, 96, 120, 160, 192,
 * 240, 320, 384, 480, 640, 768, 960 (radix 8/5/4/3/2 passes, the radix set of
 * FFTE, src/fft/ffte1/factor.f:19-43), in both precisions; PM_ERR_SIZE
 * otherwise.  The fused FP32 deposit + z FFT and the x-slab decomposition
 * need a power of two.  grad_order is 2 (the reference's 2-point centred difference,
 * src/utils/utils.cpp:115-137) or 4.  stream may be NULL (legacy default
 * stream).  Replaces the setup of src/core/main.cpp:30-81 and the FFT
 * constructor src/fft/fftw/fft.cpp:3-59 (plans, Green's table). */
int pm_plan_create(int ng, int precision, int green_kind, int grad_order, void* stream,
                   pm_plan** plan);
int pm_plan_destroy(pm_plan* plan);
/* Bytes of device memory the plan holds (workspace included). */
int pm_plan_device_bytes(const pm_plan* plan, size_t* bytes);
/* Waits for the plan's stream, then returns PM_ERR_RANGE if any kernel since
 * the last check met a bad position (and clears the flag), else PM_OK. */
int pm_plan_check(pm_plan* plan);
/* Message of the calling thread's last failed call ("" if none). */
const char* pm_last_error(void);

/* Per-kernel stage timers: the B200 form of the reference's per-stage
 * wall-clock buckets (src/utils/utils.cpp:3-20, src/core/main.cpp:88-143).
 * Launch counts per stage are always kept; with timing on, every kernel is
 * bracketed by CUDA events on the plan's stream.  pm_plan_read_timing waits
 * for the stream and fills ms[PM_STAGE_COUNT] (summed milliseconds) and
 * launches[PM_STAGE_COUNT] (either may be NULL); reset != 0 zeroes both. */
#define PM_STAGE_COUNT 19
int pm_plan_set_timing(pm_plan* plan, int on);
/* Shape of the strided FFT passes (new; the knobs the ensemble autotuner
 * turns): tile_cols kz columns per block (0 the default; 8, 16 or 32 on FP32
 * plans with ng <= 128) and the first radix of the two-pass line split (0
 * the default; FP32 plans with power-of-two ng in 16..128 also take the
 * smaller alternative, see pm_ensemble_info).  PM_ERR_ARG otherwise. */
int pm_plan_set_fft_shape(pm_plan* plan, int tile_cols, int radix1);
int pm_plan_read_timing(pm_plan* plan, double* ms, int64_t* launches, int reset);
/* Gather of pm_step_f32 (new; no counterpart in the reference):
 *   PM_GATHER_CACHED  one thread per particle in the caller's order, the 56
 *                     potential values of its stencil read through L1 (the
 *                     default; fastest when neighbouring array entries are
 *                     neighbouring particles, e.g. Lagrangian or sorted order)
 *   PM_GATHER_TILED   particles in the deposit's bin order (4 x 4-cell column
 *                     tile, face class, 64-cell z chunk), each block's stencil
 *                     region staged in shared memory: its cost does not depend
 *                     on the particle order (FP32 plans, power-of-two ng in
 *                     [256, 1024]; PM_ERR_SIZE otherwise).
 * Both give the same forces up to FP32 rounding. */
#define PM_GATHER_CACHED 0
#define PM_GATHER_TILED 1
int pm_plan_set_gather(pm_plan* plan, int mode);
/* Name of stage i ("mesh_init", "deposit", "fft_z_r2c", ...), "" if out of range. */
const char* pm_stage_name(int stage);

/* ------------------------------------------- FP64 stages (PM_FP64 plan) */

/* delta = -1 + sum_p mass * W_CIC(x_p - c), periodic; writes every cell of
 * mesh [ng][ng][ng+2] (padding set to 0).
 * Replaces init_buf, deposit_particles, reduce_private_to_shared
 * (src/utils/utils.cpp:38-113; cic_deposit include/utils/utils_inline.h:25-49),
 * TransposeSlab::execute (src/decomp/slab/transpose_slab.cpp:37-39) and
 * ReorderSlab::execute (src/decomp/slab/reorder_slab.cpp:43-68). */
int pm_deposit_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                   double mass, double* mesh);

/* In-place unnormalised R2C, sign -1: mesh -> spectrum.
 * Replaces FFT::forward (src/fft/fftw/fft.cpp:96; src/fft/ffte1/fft.cpp:61-64). */
int pm_fft_r2c_f64(pm_plan* plan, double* mesh);

/* spectrum *= G(k) / ng^3 (G per the plan's green_kind, G(0) = 0).
 * Replaces FFT::apply_green (src/fft/fftw/fft.cpp:75-82) with its table
 * (fft.cpp:50-57) computed on the fly. */
int pm_green_f64(pm_plan* plan, double* mesh, double c_poisson);

/* In-place unnormalised C2R, sign +1: spectrum -> mesh (padding zeroed; the
 * imaginary parts of kz = 0 and kz = ng/2 are ignored, as FFTW does).
 * Replaces FFT::backward (src/fft/fftw/fft.cpp:97; src/fft/ffte1/fft.cpp:65-68). */
int pm_fft_c2r_f64(pm_plan* plan, double* mesh);

/* pm_fft_r2c_f64 + pm_green_f64 + pm_fft_c2r_f64 with the x-direction
 * forward transform, Green multiply and inverse fused into one pass. */
int pm_poisson_f64(pm_plan* plan, double* mesh, double c_poisson);

/* f = -grad(phi) by the plan's finite difference, periodic.  phi is a mesh
 * [ng][ng][ng+2]; fx, fy, fz are force arrays [ng][ng][ng].
 * Replaces ReorderSlabBack::execute (src/decomp/slab/reorder_slab_back.cpp:37-49),
 * TransposeSlabBack::execute (src/decomp/slab/transpose_slab_back.cpp:47-49)
 * and centered_derivatives (src/utils/utils.cpp:115-137). */
int pm_gradient_f64(pm_plan* plan, const double* phi, double* fx, double* fy, double* fz);

/* p += c_kick * (trilinear CIC interpolation of f at x).
 * Replaces update_particles (src/utils/utils.cpp:141-170; trilerp1
 * include/utils/utils_inline.h:55-70). */
int pm_interp_kick_f64(pm_plan* plan, const double* x, const double* y, const double* z,
                       const double* fx, const double* fy, const double* fz, double* px,
                       double* py, double* pz, int64_t np, double c_kick);

/* x += dt * p, wrapped into [0, ng).  No counterpart in the reference,
 * which never moves particles (src/core/main.cpp:90-139). */
int pm_drift_f64(pm_plan* plan, double* x, double* y, double* z, const double* px,
                 const double* py, const double* pz, int64_t np, double dt);

/* One full step on the plan's own workspace: deposit, Poisson (r2c, Green,
 * c2r as separate passes), gradient, interpolate + kick, then drift by dt
 * (dt = 0: no drift, the reference's step).  The reference's stage loop body,
 * src/core/main.cpp:91-138. */
int pm_step_f64(pm_plan* plan, double* x, double* y, double* z, double* px, double* py,
                double* pz, int64_t np, double mass, double c_poisson, double c_kick, double dt);

/* ------------------------------------------------- FP64 adjoints (new)
 * Vector-Jacobian products of the step for reverse-mode differentiation; no
 * counterpart in the reference.  All add into their output arrays.
 *
 * pm_adjoint_deposit_f64: xbar += (d delta / d x)^T dbar, the adjoint of
 *   pm_deposit_f64 (dbar a mesh [ng][ng][ng+2]; padding ignored): the CIC
 *   weight-derivative gather mass * grad W(x_p - c) . dbar(c).
 * pm_adjoint_force_f64: xbar += scale * (dF/dx)^T u, F the particle forces
 *   of pm_step_f64 at x (deposit, Poisson with c_poisson, gradient,
 *   interpolation): the direct weight-derivative term u . grad W . f plus the
 *   mesh term through the transposed pairs (interpolation^T = deposit,
 *   gradient^T = -gradient, the symmetric Green's multiply, deposit^T =
 *   weight-derivative gather).  Uses the plan's workspace.
 * pm_step_adjoint_f64: the adjoint of one pm_step_f64 (v' = v + c_kick F(x);
 *   x' = x + dt v').  On entry (xbar, vbar) are the adjoints of (x', v'); on
 *   return those of (x, v).  x is the state the forward step started from. */
int pm_adjoint_deposit_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                           double mass, const double* dbar, double* xbar, double* ybar, double* zbar);
int pm_adjoint_force_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                         double mass, double c_poisson, const double* ux, const double* uy,
                         const double* uz, double scale, double* xbar, double* ybar, double* zbar);
int pm_step_adjoint_f64(pm_plan* plan, const double* x, const double* y, const double* z, int64_t np,
                        double mass, double c_poisson, double c_kick, double dt, double* xbar,
                        double* ybar, double* zbar, double* vxbar, double* vybar, double* vzbar);

/* ------------------------------------------------- FP32 adjoints (new)
 * The same vector-Jacobian products for the FP32 split-position step
 * (pm_step_f32): positions are cell + offset, the adjoint arrays are FP32
 * per particle, dbar is an FP32 mesh [ng][ng][ng+2].  No counterpart in the
 * reference.  The force Jacobian is formed from phi at the particle (no
 * force meshes); the mesh term uses a second FP32 mesh of the plan.
 * pm_step_adjoint_f32 takes the split state the forward step started from. */
int pm_adjoint_deposit_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                           const float* oz, int64_t np, float mass, const float* dbar, float* xbar,
                           float* ybar, float* zbar);
int pm_adjoint_force_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                         const float* oz, int64_t np, float mass, double c_poisson, const float* ux,
                         const float* uy, const float* uz, double scale, float* xbar, float* ybar,
                         float* zbar);
int pm_step_adjoint_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                        const float* oz, int64_t np, float mass, double c_poisson, double c_kick, double dt,
                        float* xbar, float* ybar, float* zbar, float* vxbar, float* vybar, float* vzbar);

/* ------------------------------------------- FP64 reductions (new)
 * Conserved quantities summed in FP64 whatever the plan's precision, into
 * the caller's device array out[4]: out[0] = sum over cells of (mesh + 1),
 * the total mass of a density-contrast mesh (padding ignored; 0 when mesh is
 * NULL); out[1..3] = mass * sum_p v_p, the total momentum (0 when the
 * velocity arrays are NULL).  Deterministic: the same data give the same
 * bits.  Asynchronous on the plan's stream.  No counterpart in the
 * reference. */
int pm_reduce_f32(pm_plan* plan, const float* mesh, const float* vx, const float* vy, const float* vz,
                  int64_t np, double mass, double* out);
int pm_reduce_f64(pm_plan* plan, const double* mesh, const double* vx, const double* vy, const double* vz,
                  int64_t np, double mass, double* out);

/* Device pointer to the plan's own mesh [ng][ng][ng+2] (density after the
 * deposit of pm_step_*, potential after it returns). */
int pm_plan_mesh(pm_plan* plan, void** mesh);

/* ---------------------------------- FP32 split-position path (PM_FP32 plan)
 * Positions are an integer cell plus an FP32 in-cell offset in [0, 1):
 *   cell = (ix << 20) | (iy << 10) | iz, offsets ox, oy, oz.
 * Velocities / momenta are FP32.  The drift is accumulated in FP64. */

int pm_split_positions(pm_plan* plan, const double* x, const double* y, const double* z,
                       int64_t np, uint32_t* cell, float* ox, float* oy, float* oz);
int pm_join_positions(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                      const float* oz, int64_t np, double* x, double* y, double* z);

/* FP32 counterparts of the stages above; mesh is float [ng][ng][ng+2].
 * The FP32 deposit bins the particles by 16^3-cell tile every call (counting
 * sort into plan-owned scratch: 4 bytes per particle plus 3 x 4 bytes per
 * (tile, face class) bucket) and writes each cell once from its tile's block;
 * any particle order is accepted. */
int pm_deposit_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                   const float* oz, int64_t np, float mass, float* mesh);
/* Reorders the seven particle arrays in place into Z-order of their 16^3-cell
 * tiles (counting sort; a temporary copy of the arrays is allocated and freed
 * on the plan's stream).  Only memory locality changes, never results beyond
 * rounding: call it after the particles have moved far from sorted order. */
int pm_sort_f32(pm_plan* plan, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                float* vy, float* vz, int64_t np);
int pm_fft_r2c_f32(pm_plan* plan, float* mesh);
int pm_green_f32(pm_plan* plan, float* mesh, double c_poisson);
int pm_fft_c2r_f32(pm_plan* plan, float* mesh);
int pm_poisson_f32(pm_plan* plan, float* mesh, double c_poisson);
/* Forces at the particles, gradient fused into the gather: f* [np] FP32. */
int pm_interp_f32(pm_plan* plan, const float* phi, const uint32_t* cell, const float* ox,
                  const float* oy, const float* oz, int64_t np, float* fx, float* fy, float* fz);
/* v += c_kick * force(x) then x += dt * v (FP64 accumulation, re-split);
 * gradient, interpolation, kick and drift in one pass over the particles. */
int pm_kick_drift_f32(pm_plan* plan, const float* phi, uint32_t* cell, float* ox, float* oy,
                      float* oz, float* vx, float* vy, float* vz, int64_t np, double c_kick,
                      double dt);
/* The first part of pm_step_f32: binning, the deposit fused with the z FFT
 * pass, the y / x + Green / y passes and z C2R -- the potential of the
 * particles in the plan's workspace mesh (pm_plan_mesh, [ng][ng][ng+2]).
 * pm_kick_drift_f32 on that mesh completes the step with the same result
 * as pm_step_f32 (its default gather), possibly over particle ranges: the
 * velocities are not read until then. */
int pm_potential_f32(pm_plan* plan, const uint32_t* cell, const float* ox, const float* oy,
                     const float* oz, int64_t np, float mass, double c_poisson);
/* One full FP32 step on the plan's workspace: binning by 4 x 4-cell column
 * tile, the deposit fused with the z R2C pass (power-of-two ng >= 32; the
 * tile deposit otherwise), the y / x + Green / y passes, z C2R, then
 * gradient + interpolation + kick + drift in one pass.  A cell word whose
 * indices lie outside [0, ng) is taken as the same periodic cell.  For
 * ng >= 512 this call and pm_poisson_f32 also give the plan a second half
 * spectrum (ng^2 (ng/2+1) complex, 4.3 GB at 1024) that the x + Green pass
 * writes transposed; pm_plan_device_bytes counts it. */
int pm_step_f32(pm_plan* plan, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                float* vy, float* vz, int64_t np, float mass, double c_poisson, double c_kick,
                double dt);

/* Allocation-free FP32 deposit.  No counterpart in the reference.  For
 * callers that cannot allocate device memory themselves: code under a host
 * framework whose allocator owns every device allocation, or a per-step path
 * that must not allocate.  Same result as pm_deposit_f32 (delta into mesh
 * [ng][ng][ng+2], background -1), but needs no plan and calls no cudaMalloc,
 * cudaFree or allocating library routine: its scratch is a file-scope device
 * array of 8.4 MiB (3 * 32768 + 17 bucket words plus 2^21 permutation words)
 * that every GPU loading the library holds until the process exits.
 * Limits: ng a power of two in [8, 256], np <= 2097152; larger sizes return
 * PM_ERR_SIZE.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  Every call shares the one array, which
 * keeps the previous call's contents (the counters are cleared on the stream
 * at the start of each call): calls that overlap on the GPU -- on different
 * streams, or from different threads -- race and give wrong results.
 * stream may be NULL. */
int pm_deposit_f32_noalloc(int ng, const uint32_t* cell, const float* ox, const float* oy,
                           const float* oz, int64_t np, float mass, float* mesh, void* stream);

/* ------------------------------------------ batched ensemble (FP32, new)
 * Independent periodic boxes of mixed mesh sizes advanced together; no
 * counterpart in the reference.  Particles of all boxes share the seven split
 * arrays, box b owning np[b] consecutive entries in box order (positions in
 * its own cell units).  Boxes of one mesh size form a class: every kernel of
 * the step covers the whole class in one launch, classes run concurrently on
 * their own streams.  mass[b] is box b's particle mass (host array, copied).
 * autotune != 0 picks, at creation, the shape of the strided FFT passes
 * (column-tile width x radix split) of every class with ng <= 128: whole
 * steps of all classes run concurrently, as in the run's graph, on a lattice
 * of particles in temporary device arrays (28 bytes per particle, freed
 * before the call returns), and each candidate is scored by the median of 21
 * such steps, class by class for two rounds;
 * tune_cache (may be NULL) is a
 * text file of earlier choices, read first and rewritten when new ones were
 * measured.  stream NULL: the ensemble uses its own stream (pm_ensemble_sync
 * waits for it).  Spectral / discrete Green and gradient order as for plans. */
typedef struct pm_ensemble pm_ensemble;
int pm_ensemble_create(int nbox, const int* ng, const int64_t* np, const float* mass, int green_kind,
                       int grad_order, int autotune, const char* tune_cache, void* stream,
                       pm_ensemble** ensemble);
int pm_ensemble_destroy(pm_ensemble* ensemble);
int pm_ensemble_sync(pm_ensemble* ensemble);
/* One step of every box: deposit, Poisson, kick by c_kick, drift by dt. */
int pm_ensemble_step_f32(pm_ensemble* ensemble, uint32_t* cell, float* ox, float* oy, float* oz,
                         float* vx, float* vy, float* vz, double c_poisson, double c_kick, double dt);
/* `steps` leapfrog KDK steps of every box (steps + 1 force evaluations, half
 * kicks merged), as one CUDA graph: captured on the first call and replayed
 * while the arrays, c_poisson, dt and steps stay the same. */
int pm_ensemble_run_f32(pm_ensemble* ensemble, uint32_t* cell, float* ox, float* oy, float* oz,
                        float* vx, float* vy, float* vz, double c_poisson, double dt, int steps);
/* Classes (mesh size, boxes, chosen tile width, first radix of the chosen
 * two-pass split of the strided FFT passes; 0 for the mixed-radix 48 / 96),
 * device bytes held and the node count of the last captured graph; any
 * output may be NULL. */
int pm_ensemble_info(const pm_ensemble* ensemble, int* nclasses, int* class_ng, int* class_nbox,
                     int* class_tk, int* class_radix, size_t* device_bytes, size_t* graph_nodes);

/* ------------------------------------------ x-slab decomposition (FP32)
 * One periodic ng^3 mesh split over nranks ranks (one GPU each) as x-slabs
 * of nx = ng / nranks planes, rank r owning planes [r nx, (r + 1) nx) and the
 * particles whose cell lies there (split positions as for pm_step_f32).  The
 * reference's slab layout: FFTW-MPI's local_n0 slabs (src/fft/fftw/fft.cpp:16)
 * fed by TransposeSlab + ReorderSlab (src/decomp/slab/transpose_slab.cpp:3-39,
 * reorder_slab.cpp:43-68) and read back through ReorderSlabBack +
 * TransposeSlabBack (reorder_slab_back.cpp:37-49, transpose_slab_back.cpp:3-49).
 * ng a power of two in [32, 1024]; nranks a power of two with nx a multiple
 * of 4.  The caller moves the data between ranks (NCCL, or copies between
 * slabs of one process); one step is, on every rank in the same order:
 *
 *   pm_slab_deposit_f32      deposit + z R2C into the own planes, and the +1
 *                            corners of the last plane into the ghost plane
 *   exchange A               ghost plane (buffer plane nx + 2) to rank r + 1
 *   pm_slab_fold_f32         add the ghost plane received from rank r - 1
 *   pm_slab_forward_f32      y forward; rows packed into `send`
 *   exchange B               all-to-all: block d of `send` (nx ng (ng + 2)
 *                            / nranks floats) to rank d, into block r of
 *                            `recv` on rank d
 *   pm_slab_xgreen_f32       x forward, Green, x inverse; packed into `send`
 *   exchange B again
 *   pm_slab_backward_f32     y inverse, z C2R: the potential in planes
 *                            2 .. nx + 1 of the buffer
 *   exchange C               buffer planes nx, nx + 1 to rank r + 1's planes
 *                            0, 1; planes 2, 3, 4 to rank r - 1's planes
 *                            nx + 2 .. nx + 4 (the potential halo)
 *   pm_slab_kick_drift_f32   fused gradient + gather + kick + drift
 *   pm_slab_migrate_sort     particles counted by new owner (host counts)
 *   pm_slab_migrate_pack     particles packed in owner order, W words each
 *   exchange D               counts, then the packed particles, all-to-all
 *   pm_slab_migrate_unpack   received (and kept) particles into the arrays
 *
 * The particle migration is new: the reference never moves particles. */
typedef struct pm_slab pm_slab;
int pm_slab_create(int ng, int nranks, int rank, int green_kind, int grad_order, void* stream, pm_slab** slab);
int pm_slab_destroy(pm_slab* slab);
/* Geometry and device buffers: nx own planes starting at x0; plane_floats =
 * ng (ng + 2) floats per buffer plane; buf = [nx + 6] planes (0-1 lower
 * halo, 2 .. nx + 1 own, nx + 2 ghost plane / upper halo); send and recv =
 * xfer_floats floats each.  Any output may be NULL. */
int pm_slab_info(const pm_slab* slab, int* nx, int* x0, size_t* plane_floats, void** buf, void** send, void** recv,
                 size_t* xfer_floats, size_t* device_bytes);
/* The slab's FP32 plan (stream, stage timers, pm_plan_check). */
int pm_slab_plan(pm_slab* slab, pm_plan** plan);
int pm_slab_deposit_f32(pm_slab* slab, const uint32_t* cell, const float* ox, const float* oy, const float* oz,
                        int64_t np, float mass);
int pm_slab_fold_f32(pm_slab* slab, const float* ghost);
int pm_slab_forward_f32(pm_slab* slab);
int pm_slab_xgreen_f32(pm_slab* slab, double c_poisson);
int pm_slab_backward_f32(pm_slab* slab);
/* A particle whose cell is outside the slab is clamped into it and reported
 * by pm_slab_check (PM_ERR_RANGE). */
int pm_slab_kick_drift_f32(pm_slab* slab, uint32_t* cell, float* ox, float* oy, float* oz, float* vx, float* vy,
                           float* vz, int64_t np, double c_kick, double dt);
/* counts: host array of nranks; waits for the slab's stream. */
int pm_slab_migrate_sort(pm_slab* slab, const uint32_t* cell, int64_t np, int64_t* counts);
/* arrays: host array of narrays (<= 8) device arrays of 32-bit words;
 * packed[i * narrays + w] = arrays[w][p_i], p_i in the order of the last
 * pm_slab_migrate_sort (owner rank ascending). */
int pm_slab_migrate_pack(pm_slab* slab, void* const* arrays, int narrays, int64_t np, uint32_t* packed);
/* arrays[w][at + i] = packed[i * narrays + w], i < n. */
int pm_slab_migrate_unpack(pm_slab* slab, const uint32_t* packed, int64_t n, void* const* arrays, int narrays,
                           int64_t at);
int pm_slab_check(pm_slab* slab);
/* Transposes by peer stores (new; the fused form of exchange B): the y
 * forward and the x + Green pass store each output row straight into the
 * buffer of the rank that owns it, through peer device pointers (one per
 * rank, in rank order, each xfer_floats floats and mapped into this
 * process, e.g. by pm_ipc_open), at this rank's block -- the layouts
 * exchange B would deliver.  No collective moves the spectrum; the caller
 * puts a barrier across the ranks after each of the two stores (every
 * store done before any rank reads) and before the next step's forward.
 *   pm_slab_forward_peers_f32    y forward; rows (ky, x) into peer_recv[ky / nx]
 *   pm_slab_xgreen_peers_f32     x + Green on `recv` (this rank's buffer the
 *                                forwards filled); rows into peer_rows[kx / nx]
 *   pm_slab_backward_rows_f32    y inverse from `rows` (this rank's buffer the
 *                                x + Green passes filled), z C2R
 * At most 16 ranks (PM_ERR_SIZE beyond). */
/* Peer pointers without a collective library: a buffer of this process
 * (the base of a device allocation, e.g. the `send` / `recv` of
 * pm_slab_info) exported as an opaque handle of PM_IPC_HANDLE_BYTES bytes,
 * opened in another process as a device pointer to the same memory (plain
 * CUDA IPC peer mapping, no multicast), closed when done. */
#define PM_IPC_HANDLE_BYTES 64
int pm_ipc_export(const void* dev_ptr, void* handle);
int pm_ipc_open(const void* handle, void** dev_ptr);
int pm_ipc_close(void* dev_ptr);
int pm_slab_forward_peers_f32(pm_slab* slab, void* const* peer_recv, int npeers);
int pm_slab_xgreen_peers_f32(pm_slab* slab, const void* recv, double c_poisson, void* const* peer_rows,
                             int npeers);
int pm_slab_backward_rows_f32(pm_slab* slab, const void* rows);

/* ------------------------------------- pencil decomposition (FP32, new)
 * The decomposition the reference's Makefile names (DECOMP_CHOICES "pencil",
 * Makefile:1) but does not contain; it lifts the slab path's limit of one
 * x plane block per rank.  px x py ranks, rank r = rx py + ry owning the
 * pencil x in [rx nx, (rx + 1) nx), y in [ry ny, (ry + 1) ny), all z, with
 * nx = ng / px, ny = ng / py, and the particles whose cell lies there.  ng a
 * power of two in [32, 1024]; px, py powers of two with nx, ny >= 4.  The
 * half spectrum's H = ng / 2 + 1 kz planes are split into py chunks
 * [kb(c), kb(c + 1)), kb(c) = floor(c H / py), hc(c) = kb(c + 1) - kb(c); the
 * ky axis into px chunks of nx.  A y group is the py ranks of one rx, an x
 * group the px ranks of one ry.  Buffers (complex = 2 floats):
 *   halo  [nx + 5][ny + 5][ng + 2] floats, row (x - x0 + 2, y - y0 + 2)
 *   send, recv  xfer_floats floats each
 * One step, on every rank in the same order:
 *
 *   pm_pencil_deposit_f32    CIC deposit into the halo buffer's own rows and
 *                            the +1 ghost rows x = nx, y = ny
 *   exchange A               ghost rows to the neighbours: the x ghost
 *                            (buffer rows (nx + 2, 2 .. ny + 1)) to rank
 *                            (rx + 1, ry), the y ghost ((2 .. nx + 1, ny + 2))
 *                            to (rx, ry + 1), the corner (nx + 2, ny + 2) to
 *                            (rx + 1, ry + 1); ng + 2 floats per row
 *   pm_pencil_fold_f32       add the received x ghost, y ghost and corner
 *   pm_pencil_forward_f32    z R2C; kz chunk c ([nx][ny][hc(c)]) packed into
 *                            send at complex offset nx ny kb(c)
 *   exchange B (y group)     chunk c to group member c, into recv block s
 *                            (complex offset s nx ny hc(ry)) from member s
 *   pm_pencil_yfwd_f32       y forward; ky chunk d ([nx][nx][hc(ry)]) packed
 *                            into send block d
 *   exchange C (x group)     block d to member d, into recv block s
 *   pm_pencil_xgreen_f32     x forward, Green, x inverse; send = recv
 *   exchange C again
 *   pm_pencil_yinv_f32       y inverse; y block d ([nx][ny][hc(ry)]) into
 *                            send block d (complex offset d nx ny hc(ry))
 *   exchange B reversed      block d to member d, into recv at complex
 *                            offset nx ny kb(s) from member s (hc(s) wide)
 *   pm_pencil_backward_f32   z C2R: the potential in the own rows of halo
 *   exchange D               potential halo: x rows first (own y rows),
 *                            buffer x rows nx, nx + 1 to (rx + 1, ry)'s 0, 1
 *                            and 2, 3, 4 to (rx - 1, ry)'s nx + 2 .. nx + 4;
 *                            then y rows over all nx + 5 x rows likewise
 *   pm_pencil_kick_drift_f32 gradient + gather + kick + drift
 *   pm_pencil_migrate_sort / _pack / _unpack   as for the slabs, by owner
 *                            rank rx py + ry
 */
typedef struct pm_pencil pm_pencil;
int pm_pencil_create(int ng, int px, int py, int rank, int green_kind, int grad_order, void* stream,
                     pm_pencil** pencil);
int pm_pencil_destroy(pm_pencil* pencil);
/* Geometry and device buffers; any output may be NULL. */
int pm_pencil_info(const pm_pencil* pencil, int* nx, int* ny, int* x0, int* y0, void** halo, void** send,
                   void** recv, size_t* xfer_floats, size_t* device_bytes);
int pm_pencil_plan(pm_pencil* pencil, pm_plan** plan);
int pm_pencil_deposit_f32(pm_pencil* pencil, const uint32_t* cell, const float* ox, const float* oy,
                          const float* oz, int64_t np, float mass);
/* xghost: ny rows, yghost: nx rows, corner: 1 row of ng + 2 floats each. */
int pm_pencil_fold_f32(pm_pencil* pencil, const float* xghost, const float* yghost, const float* corner);
int pm_pencil_forward_f32(pm_pencil* pencil);
int pm_pencil_yfwd_f32(pm_pencil* pencil);
int pm_pencil_xgreen_f32(pm_pencil* pencil, double c_poisson);
int pm_pencil_yinv_f32(pm_pencil* pencil);
int pm_pencil_backward_f32(pm_pencil* pencil);
/* A particle whose cell is outside the pencil is clamped into it and
 * reported by pm_pencil_check (PM_ERR_RANGE). */
int pm_pencil_kick_drift_f32(pm_pencil* pencil, uint32_t* cell, float* ox, float* oy, float* oz, float* vx,
                             float* vy, float* vz, int64_t np, double c_kick, double dt);
/* counts: host array of px py; waits for the pencil's stream. */
int pm_pencil_migrate_sort(pm_pencil* pencil, const uint32_t* cell, int64_t np, int64_t* counts);
int pm_pencil_migrate_pack(pm_pencil* pencil, void* const* arrays, int narrays, int64_t np, uint32_t* packed);
int pm_pencil_migrate_unpack(pm_pencil* pencil, const uint32_t* packed, int64_t n, void* const* arrays,
                             int narrays, int64_t at);
int pm_pencil_check(pm_pencil* pencil);
/* Transposes by peer stores (new; the fused form of exchanges B and C): each
 * pass stores its output blocks straight into the buffers of the group
 * members that own them -- peer device pointers in member order (y group:
 * member c = rank rx py + c; x group: member d = rank d py + ry), xfer_floats
 * floats each, mapped into this process -- at the block the all-to-all would
 * have filled.  Two such buffers per rank, A and B, alternate:
 *   pm_pencil_forward_peers_f32   z R2C, kz chunk c into A of y member c
 *   pm_pencil_yfwd_peers_f32      y forward of `in` (own A); ky chunk d into B
 *                                 of x member d
 *   pm_pencil_xgreen_peers_f32    x + Green of `in` (own B); x block d into A
 *                                 of x member d
 *   pm_pencil_yinv_peers_f32      y inverse of `in` (own A); y block d into B
 *                                 of y member d
 *   pm_pencil_backward_from_f32   z C2R of `in` (own B) into the halo buffer
 * The caller puts a barrier across the ranks after every store phase (and
 * before the next step's forward).  At most 16 members per group. */
int pm_pencil_forward_peers_f32(pm_pencil* pencil, void* const* peer_a, int npeers);
int pm_pencil_yfwd_peers_f32(pm_pencil* pencil, const void* in, void* const* peer_b, int npeers);
int pm_pencil_xgreen_peers_f32(pm_pencil* pencil, const void* in, double c_poisson, void* const* peer_a,
                               int npeers);
int pm_pencil_yinv_peers_f32(pm_pencil* pencil, const void* in, void* const* peer_b, int npeers);
int pm_pencil_backward_from_f32(pm_pencil* pencil, const void* in);

/* ---------------------------------------------- initial conditions (new)
 * Zel'dovich particles on an nrow^3 lattice q = (i + 1/2) ng/nrow from a
 * Gaussian random field with P(k) ~ k^n_s, scaled to an rms 3D displacement
 * of rms_cells; velocities = vel_factor * displacement.  Lagrangian order,
 * z fastest.  FP64, generated on the device (needs ~4 nrow^3 doubles of
 * temporary device memory).  The reference draws uniform positions only
 * (src/utils/utils.cpp:22-36). */
int pm_ic_zeldovich(int ng, int nrow, double n_s, double rms_cells, uint64_t seed,
                    double vel_factor, double* x, double* y, double* z, double* vx, double* vy,
                    double* vz, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* PM_B200_H */
