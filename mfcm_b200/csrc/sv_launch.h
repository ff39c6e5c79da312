// sv_launch.h -- host-callable launchers for the kernels in sv_kernels.cuh. They are
// explicitly instantiated per value type in sv_f64.cu (compiled with -fmad=false so every
// FP64 operation is separately rounded, as in the reference) and sv_f32.cu.
#pragma once
#include <cuda_runtime.h>

#include "sv_kernels.cuh"

namespace svk {

// Tile shapes compiled for the fused stage kernel (TX x TY cells per CTA, MINB resident
// CTAs per SM requested from the register allocator).
struct TileShape { int tx, ty, minb; };
constexpr TileShape kTiles[] = {{32, 8, 1}, {32, 8, 3}, {32, 4, 4}, {64, 4, 3}};
constexpr int kNumTiles = 4;

template <typename T> size_t stage_smem_bytes(int tile);
template <typename T> cudaError_t launch_stage(const StageParams<T>& P, int tile, cudaStream_t s);

// Stage-kernel variants, in two schedules:
//  fused (one pass per RK stage): 0..3 the tiled shared-memory kernel with kTiles[v]; 4..10
//   the column-sweep kernel with 16 / 32 / 64 / 32 / 32 / 32 / 32 output rows per warp, the
//   last four with register caps for 3, 4, 5 and 6 resident 4-warp blocks per SM; 12, 13
//   (FP32 only) the column sweep of 32-row strips whose interior strip pairs run two cells
//   per lane (sweep_pair_kernel), with register caps for 3 and 4 blocks per SM; 14, 15 (FP32
//   only) the one-cell sweep of 32-row strips capped for 7 and 8 blocks per SM;
//  split (two passes per RK stage): 11 the slopes pass (slopes_kernel) then the tiled 32 x 8
//   kernel at 3 CTAs/SM reading those slopes.
constexpr int kNumVariants = 16;
constexpr int kSplitVariant = 11;
constexpr int kSweepRows[7] = {16, 32, 64, 32, 32, 32, 32};
inline bool variant_is_pair(int v) { return v == 12 || v == 13; }
// variants compiled for FP32 solvers only (the two-cells-per-lane sweep, the tightest caps)
inline bool variant_is_fp32_only(int v) { return v >= 12 && v <= 15; }
inline bool variant_is_sweep(int v) { return (v >= 4 && v <= 10) || (v >= 12 && v <= 15); }
inline bool variant_is_split(int v) { return v == kSplitVariant; }
// column-sweep variants: output rows per strip (0 for the other variants)
inline int variant_sweep_rows(int v) {
  if (v >= 4 && v <= 10) return kSweepRows[v - 4];
  return (v >= 12 && v <= 15) ? 32 : 0;
}
// per-CTA (tiled) or per-warp (sweep) partial count
inline long long variant_partials(int v, long long nx, long long ny) {
  if (v == kSplitVariant) v = 1;  // the split schedule's stage pass is the tiled 32 x 8 kernel
  if (v < 4) return ((nx + kTiles[v].tx - 1) / kTiles[v].tx) * ((ny + kTiles[v].ty - 1) / kTiles[v].ty);
  const long long ty = variant_sweep_rows(v);
  return ((nx + kSweepOut - 1) / kSweepOut) * ((ny + ty - 1) / ty);
}
template <typename T> cudaError_t launch_variant(const StageParams<T>& P, int variant, cudaStream_t s);
// per-strip interior flags of the column sweep with `ty` output rows (strip_flags_kernel)
template <typename T> cudaError_t launch_strip_flags(const T* z, int nx, int ny, int ty, long long nstrips,
                                                     unsigned char* flags, cudaStream_t s);
template <typename T> cudaError_t launch_bed_slopes(const T* z, int nx, int ny, double dx, double dy, T* zx, T* zy,
                                                    cudaStream_t s);
// FP64 <-> T conversion of a field on the device
template <typename T> cudaError_t launch_from_f64(const double* src, T* dst, long long n, cudaStream_t s);
template <typename T> cudaError_t launch_to_f64(const T* src, double* dst, long long n, cudaStream_t s);
// *flag = 1 when T(src[i]) differs bit for bit from ref[i] for some i (flag left as it was otherwise)
template <typename T> cudaError_t launch_differs(const double* src, const T* ref, long long n, int* flag, cudaStream_t s);
// FP32 with tile datums, from an FP64 bed on the device: the tile datums, the FP32 offsets and
// the bed slopes (FP64, rounded once); and the absolute FP64 bed back from the offsets
cudaError_t launch_datum_bed(const double* z, int nx, int ny, double dx, double dy, int dtiles_x, int dtiles_y,
                             double* zdat, float* off, float* zx, float* zy, cudaStream_t s);
cudaError_t launch_datum_absolute(const float* off, int nx, int ny, int dtiles_x, const double* zdat, double* z,
                                  cudaStream_t s);
template <typename T> cudaError_t launch_volume(const T* h, int nx, int ny, double area, double* part, int tile,
                                                cudaStream_t s);
template <typename T> cudaError_t launch_debug(const StageParams<T>& P, const DebugParams<T>& D, T* nh, T* sf,
                                               cudaStream_t s);
// batched launches: every tile of every instance (tiled 32 x 8 kernel, 3 CTAs/SM); p2 when
// every instance's dx and dy are powers of two, eddy when any instance has eddy viscosity
template <typename T> cudaError_t launch_stage_batch(const StageParams<T>* Ps, const long long* tile_start, int ninst,
                                                     long long total_tiles, bool p2, bool eddy, cudaStream_t s);
// batches of FP64 instances use the tiled variant 1; FP32 batches the column sweep of
// variant 8 (launch_sweep_batch), the fastest single-solver kernels of each precision
template <typename T> constexpr int batch_variant() { return sizeof(T) == 8 ? 1 : 8; }
template <typename T> cudaError_t launch_sweep_batch(const StageParams<T>* Ps, const long long* warp_start, int ninst,
                                                     long long total_warps, bool p2, bool eddy, cudaStream_t s);
// persistent batch kernel (persist_batch_kernel), cooperative launch filling the device
template <typename T> cudaError_t launch_persist(const PersistParams<T>& PP, bool p2, bool eddy, cudaStream_t s);
cudaError_t launch_persist_init(const FinalizeParams* Fs, PersistMember* mem, const long long* warp_start, int nact,
                                cudaStream_t s);
cudaError_t launch_finalize(const FinalizeParams& F, cudaStream_t s);
cudaError_t launch_finalize_batch(const FinalizeParams* Fs, int ninst, cudaStream_t s);
cudaError_t launch_begin_queue(const FinalizeParams* Fs, int n, cudaStream_t s);
cudaError_t launch_gather_done(Ctl* const* ctls, int n, int* done, cudaStream_t s);
cudaError_t launch_sum(const double* p, long long n, double* out, cudaStream_t s);
cudaError_t launch_accept(Ctl* ctl, cudaStream_t s);
cudaError_t launch_begin_step(Ctl* ctl, int new_step, long long budget, cudaStream_t s);

}  // namespace svk
