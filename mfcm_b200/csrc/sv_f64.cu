// sv_f64.cu -- FP64 instantiation of the stage kernels. Compiled with -fmad=false: every
// FP64 multiply and add is rounded separately, as in the reference's CPU arithmetic, which
// is what makes the FP64 path bit-identical to the oracle. (Explicit fma() calls are kept:
// they implement the exact constant-divisor division in sv_device.cuh.)
#define SV_T double
#define SV_DEFINE_COMMON_KERNELS
#include "sv_inst.cuh"

namespace svk {

cudaError_t launch_finalize(const FinalizeParams& F, cudaStream_t s) {
  finalize_kernel<1024><<<1, 1024, 0, s>>>(F);
  return cudaGetLastError();
}
cudaError_t launch_finalize_batch(const FinalizeParams* Fs, int ninst, cudaStream_t s) {
  if (ninst <= 0) return cudaSuccess;
  finalize_batch_kernel<1024><<<ninst, 1024, 0, s>>>(Fs);
  return cudaGetLastError();
}
cudaError_t launch_begin_queue(const FinalizeParams* Fs, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  begin_queue_kernel<<<(n + 127) / 128, 128, 0, s>>>(Fs, n);
  return cudaGetLastError();
}
cudaError_t launch_gather_done(Ctl* const* ctls, int n, int* done, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  gather_done_kernel<<<(n + 127) / 128, 128, 0, s>>>(ctls, n, done);
  return cudaGetLastError();
}
cudaError_t launch_sum(const double* p, long long n, double* out, cudaStream_t s) {
  sum_kernel<1024><<<1, 1024, 0, s>>>(p, n, out);
  return cudaGetLastError();
}
cudaError_t launch_accept(Ctl* ctl, cudaStream_t s) {
  accept_kernel<<<1, 1, 0, s>>>(ctl);
  return cudaGetLastError();
}
// In this unit (no contraction) so that the FP64 slopes round like those of the FP64 solver.
cudaError_t launch_datum_bed(const double* z, int nx, int ny, double dx, double dy, int dtiles_x, int dtiles_y,
                             double* zdat, float* off, float* zx, float* zy, cudaStream_t s) {
  const long long n = (long long)nx * ny, nt = (long long)dtiles_x * dtiles_y;
  if (n <= 0) return cudaSuccess;
  datum_tiles_kernel<<<unsigned((nt + 7) / 8), 256, 0, s>>>(z, nx, ny, dtiles_x, dtiles_y, zdat);
  datum_offsets_kernel<<<elementwise_blocks(n), 256, 0, s>>>(z, nx, ny, dtiles_x, zdat, off);
  bed_slopes_kernel<double, float><<<unsigned((n + 255) / 256), 256, 0, s>>>(z, nx, ny, dx, dy, zx, zy);
  return cudaGetLastError();
}
cudaError_t launch_datum_absolute(const float* off, int nx, int ny, int dtiles_x, const double* zdat, double* z,
                                  cudaStream_t s) {
  const long long n = (long long)nx * ny;
  if (n <= 0) return cudaSuccess;
  datum_absolute_kernel<<<elementwise_blocks(n), 256, 0, s>>>(off, nx, ny, dtiles_x, zdat, z);
  return cudaGetLastError();
}
cudaError_t launch_persist_init(const FinalizeParams* Fs, PersistMember* mem, const long long* warp_start, int nact,
                                cudaStream_t s) {
  if (nact <= 0) return cudaSuccess;
  persist_init_kernel<<<(nact + 127) / 128, 128, 0, s>>>(Fs, mem, warp_start, nact);
  return cudaGetLastError();
}
cudaError_t launch_begin_step(Ctl* ctl, int new_step, long long budget, cudaStream_t s) {
  begin_step_kernel<<<1, 1, 0, s>>>(ctl, new_step, budget);
  return cudaGetLastError();
}

}  // namespace svk
