// Host-runtime internals of librsgpu (not part of the C ABI).
#pragma once
#include <cstdarg>
#include <cstddef>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "rsgpu_kernels.h"

namespace rsgpu {

// thread-local last-error text behind rsgpu_last_error()
void set_error(const char *fmt, ...);

void pml_tables_host(int lpml, double dt, int prec, void *out);
int stagger_host(int physics, int nx, int ny, int nz, int l, int fs, int prec, const void *vp, const void *vs,
                 const void *rho, void *const *out);
template <typename T>
int stagger_e3d_host(int nx, int ny, int nz, int l, int fs, const T *vp, const T *vs, const T *rho, T *const *out);
void coef_table_host(int prec, double dx, double dz, std::vector<unsigned char> &out);
bool encode_field_map_host(void *map, void *base, int prec, int pitch, int rows, int boxw, int boxh);

// Device memory of plans and drivers: a library-owned stream-ordered pool per
// device that keeps up to 8 GiB of freed blocks mapped, so that creating and
// destroying a plan per call (rsgpu_modelling, rsgpu_fwi_gradient) does not map and
// unmap its arena every time.  dev_alloc returns memory usable at once by any
// stream and by synchronous copies; dev_free releases it in `st`'s order.
cudaError_t dev_alloc(void **p, size_t bytes, cudaStream_t st);
void dev_free(void *p, cudaStream_t st);
// Return the cached blocks of the current device's pool to the driver.
cudaError_t dev_trim();
void make_map_host(int dim, int prec, int ntr, const double *coords, const int *n, const double *o, const double *d,
                   const double *gshift, int *map, void *shift);

// Griewank binomial checkpoint schedule (reference: lib/revolve.cpp:31-305).
class RevolveSchedule {
public:
    RevolveSchedule(int steps, int snaps);
    int next();             // returns an RSGPU_ADVANCE.. action code
    int capo() const { return capo_; }
    int check() const { return check_; }
    int snaps() const { return snaps_; }
    int info() const { return info_; }
    static int numforw(int steps, int snaps);
    static int adjust(int steps);

private:
    static int maxrange(int ss, int tt);
    int check_, capo_, fine_, steps_, snaps_, info_;
    int turn_, reps_, range_, oldsnaps_, oldfine_;
    int ch_[512];
};

}  // namespace rsgpu
