// C entry points over the reference's own CPU kernels, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libpmref.so.
//
// TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
// reference / cpu_baseline legs load this library as the checker or as the
// timed CPU baseline; the product never links it.
//
// Every function forwards to the reference symbol named beside it; nothing
// here re-implements reference arithmetic.
#include <vector>
#include <array>
#include <omp.h>
#include "utils.h"              // include/utils/utils.h
#include "reorder_slab.h"       // include/decomp/slab/reorder_slab.h
#include "reorder_slab_back.h"  // include/decomp/slab/reorder_slab_back.h

extern "C" {

void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_max_threads(void) { return omp_get_max_threads(); }

// src/utils/utils.cpp:22-36
void ref_init_particles(double* x, double* y, double* z, size_t np, int x0, int y0, int z0,
                        int nx_loc, int ny_loc, int nz_loc, int rank) {
    init_particles(x, y, z, np, x0, y0, z0, nx_loc, ny_loc, nz_loc, rank);
}

// src/utils/utils.cpp:38-68
void ref_init_buf(double* buf, int nx, int ny, int nz, size_t ncell_local, int nthreads) {
    init_buf(buf, nx, ny, nz, ncell_local, nthreads);
}

// src/utils/utils.cpp:70-102 (cic_deposit: include/utils/utils_inline.h:25-49)
void ref_deposit_particles(const double* x, const double* y, const double* z, size_t np,
                           double* buf, size_t ncell_local, int nx, int ny, int nz,
                           int x0, int y0, int z0, double mass) {
    deposit_particles(x, y, z, np, buf, ncell_local, nx, ny, nz, x0, y0, z0, mass);
}

// src/utils/utils.cpp:104-113
void ref_reduce_private_to_shared(double* buf, size_t ncell_local, int nthreads) {
    reduce_private_to_shared(buf, ncell_local, nthreads);
}

// src/utils/utils.cpp:115-137
void ref_centered_derivatives(const double* in, double* dx, double* dy, double* dz,
                              int nx1, int ny1, int nz1) {
    centered_derivatives(in, dx, dy, dz, nx1, ny1, nz1);
}

// src/utils/utils.cpp:141-170 (trilerp1: include/utils/utils_inline.h:55-70)
void ref_update_particles(const double* x, const double* y, const double* z,
                          const double* dx, const double* dy, const double* dz,
                          double* px, double* py, double* pz, double a, size_t np,
                          int ny, int nz, int x0, int y0, int z0) {
    update_particles(x, y, z, dx, dy, dz, px, py, pz, a, np, ny, nz, x0, y0, z0);
}

// include/utils/utils_inline.h:51-53
double ref_function_a(double a) { return function_a(a); }

// include/utils/utils_inline.h:13-17
void ref_constants(double* out6) {
    out6[0] = Omega_0; out6[1] = Omega_m; out6[2] = Omega_lambda;
    out6[3] = Omega_k; out6[4] = Da; out6[5] = Start_a;
}

// src/decomp/slab/reorder_slab.cpp:3-41 (ctor) and :43-68 (execute)
void* ref_reorder_slab_create(int Ng, int ny, int nz, long local_n0, int stride,
                              const int* recvcounts, const int* rdispls, int nranks,
                              const int* dims) {
    std::vector<int> rc(recvcounts, recvcounts + nranks), rd(rdispls, rdispls + nranks);
    std::array<int, 3> d = {dims[0], dims[1], dims[2]};
    return new ReorderSlab(Ng, ny, nz, (ptrdiff_t)local_n0, stride, rc, rd, d);
}
void ref_reorder_slab_execute(void* h, const double* in, double* out) {
    static_cast<ReorderSlab*>(h)->execute(in, out);
}
void ref_reorder_slab_destroy(void* h) { delete static_cast<ReorderSlab*>(h); }

// src/decomp/slab/reorder_slab_back.cpp:3-35 (ctor) and :37-49 (execute)
void* ref_reorder_slab_back_create(int Ng, int ny_loc, int nz_loc, int stride, const int* dims,
                                   long local_n0) {
    std::array<int, 3> d = {dims[0], dims[1], dims[2]};
    return new ReorderSlabBack(Ng, ny_loc, nz_loc, stride, d, (ptrdiff_t)local_n0);
}
void ref_reorder_slab_back_execute(void* h, const double* in, double* out) {
    static_cast<ReorderSlabBack*>(h)->execute(in, out);
}
void ref_reorder_slab_back_destroy(void* h) { delete static_cast<ReorderSlabBack*>(h); }

}  // extern "C"
