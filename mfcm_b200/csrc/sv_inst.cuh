// sv_inst.cuh -- launcher definitions, included once per value type by sv_f64.cu / sv_f32.cu
// with SV_T defined to the value type.
#pragma once
#include <atomic>
#include <cmath>
#include <utility>

#include "sv_launch.h"

namespace svk {

// cudaFuncSetAttribute applies to the device that is current when it is called, so the
// opt-in to more than 48 KB of dynamic shared memory is made once per device and kernel.
// `done` is a per-kernel table indexed by device number.
constexpr int kMaxAttrDevices = 64;
template <typename K>
static cudaError_t smem_optin(K kernel, int bytes, std::atomic<bool> (&done)[kMaxAttrDevices]) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxAttrDevices && done[dev].load(std::memory_order_acquire)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < kMaxAttrDevices) done[dev].store(true, std::memory_order_release);
  return cudaSuccess;
}

// dx and dy both powers of two: the mesh divisions are exact multiplies
inline bool pow2_mesh(double dx, double dy) {
  int e;
  return std::frexp(dx, &e) == 0.5 && std::frexp(dy, &e) == 0.5;
}

template <typename T, int TX, int TY, int MINB, bool P2, bool EDDY, bool PRE = false>
static cudaError_t launch_stage_p(const StageParams<T>& P, cudaStream_t s) {
  using SM = StageSmem<T, TX, TY>;
  static std::atomic<bool> attr_set[kMaxAttrDevices];
  cudaError_t e = smem_optin(stage_kernel<T, TX, TY, MINB, P2, EDDY, PRE>, int(sizeof(SM)), attr_set);
  if (e != cudaSuccess) return e;
  dim3 grid((P.nx + TX - 1) / TX, (P.ny + TY - 1) / TY);
  stage_kernel<T, TX, TY, MINB, P2, EDDY, PRE><<<grid, TX * TY, sizeof(SM), s>>>(P);
  return cudaGetLastError();
}

// split schedule: the slopes pass, then the tiled 32 x 8 stage kernel reading its slopes
template <typename T> static cudaError_t launch_split_t(const StageParams<T>& P, cudaStream_t s) {
  const bool p2 = pow2_mesh(P.dx, P.dy);
  const long long n = (long long)P.nx * P.ny;
  const unsigned blocks = unsigned((n + 255) / 256);
  if (p2) slopes_kernel<T, true><<<blocks, 256, 0, s>>>(P);
  else slopes_kernel<T, false><<<blocks, 256, 0, s>>>(P);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (P.eddy)
    return p2 ? launch_stage_p<T, 32, 8, 3, true, true, true>(P, s) : launch_stage_p<T, 32, 8, 3, false, true, true>(P, s);
  return p2 ? launch_stage_p<T, 32, 8, 3, true, false, true>(P, s) : launch_stage_p<T, 32, 8, 3, false, false, true>(P, s);
}
// kernels compiled with the eddy-viscosity term run only for solvers that have it
template <typename T, int TX, int TY, int MINB> static cudaError_t launch_stage_t(const StageParams<T>& P, cudaStream_t s) {
  const bool p2 = pow2_mesh(P.dx, P.dy);
  if (P.eddy)
    return p2 ? launch_stage_p<T, TX, TY, MINB, true, true>(P, s) : launch_stage_p<T, TX, TY, MINB, false, true>(P, s);
  return p2 ? launch_stage_p<T, TX, TY, MINB, true, false>(P, s) : launch_stage_p<T, TX, TY, MINB, false, false>(P, s);
}

template <> size_t stage_smem_bytes<SV_T>(int tile) {
  switch (tile) {
    case 0: return sizeof(StageSmem<SV_T, 32, 8>);
    case 1: return sizeof(StageSmem<SV_T, 32, 8>);
    case 2: return sizeof(StageSmem<SV_T, 32, 4>);
    default: return sizeof(StageSmem<SV_T, 64, 4>);
  }
}

template <> cudaError_t launch_stage<SV_T>(const StageParams<SV_T>& P, int tile, cudaStream_t s) {
  switch (tile) {
    case 0: return launch_stage_t<SV_T, 32, 8, 1>(P, s);
    case 1: return launch_stage_t<SV_T, 32, 8, 3>(P, s);
    case 2: return launch_stage_t<SV_T, 32, 4, 4>(P, s);
    default: return launch_stage_t<SV_T, 64, 4, 3>(P, s);
  }
}

// A sweep launch of a stage after the first: allowed to start while the one before it runs
// (programmatic dependent launch; the sweeps of one stage touch disjoint outputs)
template <typename... KArgs, typename... Args>
static cudaError_t launch_overlapped(void (*kern)(KArgs...), dim3 grid, dim3 block, cudaStream_t s, bool overlap,
                                     Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = overlap ? attr : nullptr;
  cfg.numAttrs = overlap ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <typename T, int TY, int MINB, bool PAIR = false>
static cudaError_t launch_sweep_t(const StageParams<T>& P, int variant, cudaStream_t s) {
  constexpr int WPB = 4;
  const long long ntiles = variant_partials(variant, P.nx, P.ny);
  dim3 block(32, WPB);
  const bool p2 = pow2_mesh(P.dx, P.dy);
  bool overlap = false;  // the first launch of the stage waits for the previous stage
  cudaError_t e = cudaSuccess;
  // the general sweep over the edge and coded-out strips (every strip without lists) first:
  // few warps, each slower than an interior one, so it runs beside the interior launches
  const long long ngen = P.bstrips ? P.n_bstrips : ntiles;
  if (ngen > 0) {
    dim3 grid(unsigned((ngen + WPB - 1) / WPB));
    void (*k)(const StageParams<T>) =
        P.eddy ? (p2 ? sweep_kernel<T, TY, WPB, MINB, true, true> : sweep_kernel<T, TY, WPB, MINB, false, true>)
               : (p2 ? sweep_kernel<T, TY, WPB, MINB, true, false> : sweep_kernel<T, TY, WPB, MINB, false, false>);
    e = launch_overlapped(k, grid, block, s, overlap, P);
    if (e != cudaSuccess) return e;
    overlap = true;
  }
  // interior strip pairs (FP32, if listed) two cells per lane
  if constexpr (PAIR && sizeof(T) == 4) {
    if (P.ipairs && P.n_ipairs > 0) {
      dim3 grid(unsigned((P.n_ipairs + WPB - 1) / WPB));
      void (*k)(const StageParams<float>) =
          P.eddy ? (p2 ? sweep_pair_kernel<TY, WPB, MINB, true, true> : sweep_pair_kernel<TY, WPB, MINB, false, true>)
                 : (p2 ? sweep_pair_kernel<TY, WPB, MINB, true, false> : sweep_pair_kernel<TY, WPB, MINB, false, false>);
      e = launch_overlapped(k, grid, block, s, overlap, P);
      if (e != cudaSuccess) return e;
      overlap = true;
    }
  }
  // interior strips (if listed) in the interior kernel
  if (P.istrips && P.n_istrips > 0) {
    dim3 grid(unsigned((P.n_istrips + WPB - 1) / WPB));
    void (*k)(const StageParams<T>) =
        P.eddy ? (p2 ? sweep_interior_kernel<T, TY, WPB, MINB, true, true>
                     : sweep_interior_kernel<T, TY, WPB, MINB, false, true>)
               : (p2 ? sweep_interior_kernel<T, TY, WPB, MINB, true, false>
                     : sweep_interior_kernel<T, TY, WPB, MINB, false, false>);
    e = launch_overlapped(k, grid, block, s, overlap, P);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

// the FP32-only variants: two cells per lane with register caps for 3 and 4 blocks per SM
// (12, 13), one cell per lane capped for 7 and 8 blocks per SM (14, 15); 32-row strips
template <typename T> static cudaError_t v12_15(const StageParams<T>& P, int variant, cudaStream_t s) {
  if constexpr (sizeof(T) == 4) {
    switch (variant) {
      case 12: return launch_sweep_t<T, 32, 3, true>(P, variant, s);
      case 13: return launch_sweep_t<T, 32, 4, true>(P, variant, s);
      case 14: return launch_sweep_t<T, 32, 7>(P, variant, s);
      default: return launch_sweep_t<T, 32, 8>(P, variant, s);
    }
  }
  return cudaErrorInvalidValue;
}

template <> cudaError_t launch_variant<SV_T>(const StageParams<SV_T>& P, int variant, cudaStream_t s) {
  switch (variant) {
    case 4: return launch_sweep_t<SV_T, 16, 1>(P, variant, s);
    case 5: return launch_sweep_t<SV_T, 32, 1>(P, variant, s);
    case 6: return launch_sweep_t<SV_T, 64, 1>(P, variant, s);
    case 7: return launch_sweep_t<SV_T, 32, 3>(P, variant, s);
    case 8: return launch_sweep_t<SV_T, 32, 4>(P, variant, s);
    case 9: return launch_sweep_t<SV_T, 32, 5>(P, variant, s);
    case 10: return launch_sweep_t<SV_T, 32, 6>(P, variant, s);
    case kSplitVariant: return launch_split_t<SV_T>(P, s);
    case 12:
    case 13:
    case 14:
    case 15:
      if (sizeof(SV_T) != 4) return cudaErrorInvalidValue;  // FP32-only variants
      return v12_15<SV_T>(P, variant, s);
    default: return launch_stage<SV_T>(P, variant, s);
  }
}

template <> cudaError_t launch_strip_flags<SV_T>(const SV_T* z, int nx, int ny, int ty, long long nstrips,
                                                 unsigned char* flags, cudaStream_t s) {
  if (nstrips <= 0) return cudaSuccess;
  strip_flags_kernel<SV_T><<<unsigned((nstrips + 7) / 8), 256, 0, s>>>(z, nx, ny, ty, nstrips, flags);
  return cudaGetLastError();
}

template <> cudaError_t launch_bed_slopes<SV_T>(const SV_T* z, int nx, int ny, double dx, double dy, SV_T* zx,
                                                SV_T* zy, cudaStream_t s) {
  long long n = (long long)nx * ny;
  bed_slopes_kernel<SV_T><<<unsigned((n + 255) / 256), 256, 0, s>>>(z, nx, ny, dx, dy, zx, zy);
  return cudaGetLastError();
}

static unsigned elementwise_blocks(long long n) {
  const long long b = (n + 255) / 256;
  return unsigned(b < 148 * 16 ? (b > 0 ? b : 1) : 148 * 16);  // grid-stride beyond 16 blocks per SM
}
template <> cudaError_t launch_from_f64<SV_T>(const double* src, SV_T* dst, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  convert_kernel<double, SV_T><<<elementwise_blocks(n), 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}
template <> cudaError_t launch_differs<SV_T>(const double* src, const SV_T* ref, long long n, int* flag,
                                             cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  differs_kernel<SV_T><<<elementwise_blocks(n), 256, 0, s>>>(src, ref, n, flag);
  return cudaGetLastError();
}
template <> cudaError_t launch_to_f64<SV_T>(const SV_T* src, double* dst, long long n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  convert_kernel<SV_T, double><<<elementwise_blocks(n), 256, 0, s>>>(src, dst, n);
  return cudaGetLastError();
}

template <typename T, int TX, int TY, int MINB, bool P2, bool EDDY>
static cudaError_t launch_stage_batch_p(const StageParams<T>* Ps, const long long* tile_start, int ninst,
                                        long long total_tiles, cudaStream_t s) {
  using SM = StageSmem<T, TX, TY>;
  static std::atomic<bool> attr_set[kMaxAttrDevices];
  cudaError_t e = smem_optin(stage_batch_kernel<T, TX, TY, MINB, P2, EDDY>, int(sizeof(SM)), attr_set);
  if (e != cudaSuccess) return e;
  if (total_tiles <= 0) return cudaSuccess;
  stage_batch_kernel<T, TX, TY, MINB, P2, EDDY><<<unsigned(total_tiles), TX * TY, sizeof(SM), s>>>(Ps, tile_start,
                                                                                                     ninst);
  return cudaGetLastError();
}

template <> cudaError_t launch_stage_batch<SV_T>(const StageParams<SV_T>* Ps, const long long* tile_start, int ninst,
                                                 long long total_tiles, bool p2, bool eddy, cudaStream_t s) {
  if (eddy)
    return p2 ? launch_stage_batch_p<SV_T, 32, 8, 3, true, true>(Ps, tile_start, ninst, total_tiles, s)
              : launch_stage_batch_p<SV_T, 32, 8, 3, false, true>(Ps, tile_start, ninst, total_tiles, s);
  return p2 ? launch_stage_batch_p<SV_T, 32, 8, 3, true, false>(Ps, tile_start, ninst, total_tiles, s)
            : launch_stage_batch_p<SV_T, 32, 8, 3, false, false>(Ps, tile_start, ninst, total_tiles, s);
}

template <> cudaError_t launch_sweep_batch<SV_T>(const StageParams<SV_T>* Ps, const long long* warp_start, int ninst,
                                                 long long total_warps, bool p2, bool eddy, cudaStream_t s) {
  constexpr int WPB = 4, TY = 32, MINB = 4;  // variant 8
  if (total_warps <= 0) return cudaSuccess;
  dim3 block(32, WPB);
  dim3 grid(unsigned((total_warps + WPB - 1) / WPB));
  if (eddy) {
    if (p2) sweep_batch_kernel<SV_T, TY, WPB, MINB, true, true><<<grid, block, 0, s>>>(Ps, warp_start, ninst);
    else sweep_batch_kernel<SV_T, TY, WPB, MINB, false, true><<<grid, block, 0, s>>>(Ps, warp_start, ninst);
  } else {
    if (p2) sweep_batch_kernel<SV_T, TY, WPB, MINB, true, false><<<grid, block, 0, s>>>(Ps, warp_start, ninst);
    else sweep_batch_kernel<SV_T, TY, WPB, MINB, false, false><<<grid, block, 0, s>>>(Ps, warp_start, ninst);
  }
  return cudaGetLastError();
}

// Persistent batch kernel: one cooperative launch with as many 4-warp blocks as fit on the
// device at once (every block resident, so warps that wait for another warp's work always
// see it done).
template <> cudaError_t launch_persist<SV_T>(const PersistParams<SV_T>& PP, bool p2, bool eddy, cudaStream_t s) {
  void (*kern)(const PersistParams<SV_T>) =
      eddy ? (p2 ? persist_batch_kernel<SV_T, true, true> : persist_batch_kernel<SV_T, false, true>)
           : (p2 ? persist_batch_kernel<SV_T, true, false> : persist_batch_kernel<SV_T, false, false>);
  int dev = 0, nsm = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kPersistWarps, 0);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
  PersistParams<SV_T> arg = PP;
  void* args[] = {&arg};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(unsigned(per_sm * nsm)), dim3(32, kPersistWarps), args,
                                     0, s);
}

template <typename T, int TX, int TY>
static cudaError_t launch_volume_t(const T* h, int nx, int ny, double area, double* part, cudaStream_t s) {
  dim3 grid((nx + TX - 1) / TX, (ny + TY - 1) / TY);
  volume_partials_kernel<T, TX, TY><<<grid, TX * TY, 0, s>>>(h, nx, ny, area, part);
  return cudaGetLastError();
}

template <> cudaError_t launch_volume<SV_T>(const SV_T* h, int nx, int ny, double area, double* part, int tile,
                                            cudaStream_t s) {
  (void)tile;  // one fixed decomposition: the volume must not depend on the stage-kernel variant
  return launch_volume_t<SV_T, 32, 8>(h, nx, ny, area, part, s);
}

template <> cudaError_t launch_debug<SV_T>(const StageParams<SV_T>& P, const DebugParams<SV_T>& D, SV_T* nh,
                                           SV_T* sf, cudaStream_t s) {
  long long n = (long long)D.nx * D.ny;
  long long nf = (long long)(D.nx + 1) * D.ny + (long long)(D.ny + 1) * D.nx;
  debug_slopes_kernel<SV_T><<<unsigned((n + 255) / 256), 256, 0, s>>>(D);
  debug_flux_kernel<SV_T><<<unsigned((nf + 255) / 256), 256, 0, s>>>(D);
  debug_cell_kernel<SV_T><<<unsigned((n + 255) / 256), 256, 0, s>>>(P, D, nh, sf);
  return cudaGetLastError();
}

}  // namespace svk
