// kernels_dispatch.cu -- the unqualified kernel launchers of fargo_internal.h:
// each forwards to the kernel set of the batch's precision mode, fargo_k
// (fused multiply-adds where the compiler contracts, as the reference's
// build) or fargo_k_nofma (no contraction: the accurate mode).
#include "fargo_internal.h"

#define FARGO_BY_MODE(b, call)  \
  do {                          \
    if ((b).accurate)           \
      fargo_k_nofma::call;      \
    else                        \
      fargo_k::call;            \
  } while (0)

cudaError_t fargo_kernel_attributes(int max_nsec) {
  cudaError_t e = fargo_k::fargo_kernel_attributes(max_nsec);
  return e != cudaSuccess ? e : fargo_k_nofma::fargo_kernel_attributes(max_nsec);
}
void fargo_launch_dt_begin(const BatchDev& b, cudaStream_t s) { FARGO_BY_MODE(b, fargo_launch_dt_begin(b, s)); }
void fargo_launch_cs_refresh(const BatchDev& b, int only_disk, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_cs_refresh(b, only_disk, s));
}
void fargo_launch_cs_isothermal(const BatchDev& b, int only_disk, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_cs_isothermal(b, only_disk, s));
}
void fargo_launch_substep(const BatchDev& b, cudaGraphConditionalHandle h, int use_handle, cudaStream_t s,
                          int max_nsec, long long* launches, cudaEvent_t* ev, int part) {
  FARGO_BY_MODE(b, fargo_launch_substep(b, h, use_handle, s, max_nsec, launches, ev, part));
}
void fargo_launch_stripe_block(const BatchDev& b, double* out, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_stripe_block(b, out, s));
}
int fargo_launch_stripe_finish(const BatchDev& b, const double* blk, int nstripe, int stride, cudaStream_t s) {
  return b.accurate ? fargo_k_nofma::fargo_launch_stripe_finish(b, blk, nstripe, stride, s)
                    : fargo_k::fargo_launch_stripe_finish(b, blk, nstripe, stride, s);
}
const char* fargo_substep_kernel_name(int k) { return fargo_k::fargo_substep_kernel_name(k); }
void fargo_launch_sector_tables(const BatchDev& b, int max_nsec, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_sector_tables(b, max_nsec, s));
}
void fargo_launch_init_velocities(const BatchDev& b, int disk, long long ncell_ghost, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_init_velocities(b, disk, ncell_ghost, s));
}
void fargo_launch_disk_force(const BatchDev& b, int disk, float x, float y, float rs, float rh, float a,
                             double* out44, int nblocks, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_disk_force(b, disk, x, y, rs, rh, a, out44, nblocks, s));
}
void fargo_launch_diagnostics(const BatchDev& b, int disk, double* out3, int nblocks, cudaStream_t s) {
  FARGO_BY_MODE(b, fargo_launch_diagnostics(b, disk, out3, nblocks, s));
}
int fargo_substep_launches(const BatchDev& b) { return fargo_k::fargo_substep_launches(b); }
// both sets share their launch bounds, so one set's occupancy sizes the grids
cudaError_t fargo_size_grids(BatchDev& b, int nsm, long long ncell_tiles, int nitems) {
  return fargo_k::fargo_size_grids(b, nsm, ncell_tiles, nitems);
}
const void* fargo_cfl_kernel(int max_body) { return fargo_k::fargo_cfl_kernel(max_body); }
void fargo_launch_transport(const BatchDev& b, cudaStream_t s) { FARGO_BY_MODE(b, fargo_launch_transport(b, s)); }
