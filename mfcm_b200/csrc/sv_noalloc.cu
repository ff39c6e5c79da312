// sv_noalloc.cu -- one FP64 Runge-Kutta timestep on caller-owned device buffers, with all
// working memory taken from a fixed array compiled into this library.
//
// Who needs it: a caller that must not allocate device memory after it has started -- for
// example a coupled catchment model whose host framework owns every device allocation
// through its own pool and hands the solver only pre-allocated buffers, or a real-time
// forecasting loop where a cudaMalloc would synchronise the device and stall other work on
// it. sv_create allocates the solver's state, stage and reduction buffers; this entry point
// allocates nothing.
//
// Working memory: g_sv_scratch below, a file-scope device array of kScratchBytes. Every GPU
// that loads this library holds one copy of it until the process exits. It bounds the mesh
// to kMaxCells cells (256 x 256); larger meshes are rejected with SV_E_LIMIT.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/sv.h"
#include "sv_launch.h"
#include "sv_tableau.h"

namespace svh {
void set_global_error(const std::string& msg);
}

namespace {

constexpr long long kMaxCells = 65536;  // 256 x 256
// partial-sum slots of the 32 x 8 tiled stage kernel: at most 8192 CTAs for any mesh of at
// most kMaxCells cells (reached by a 1-cell-wide strip), times 3 + 3 * 4 stages
constexpr long long kMaxBlocks = 8192;
constexpr int kVariant = 1;  // tiled stage kernel, 32 x 8 cells per CTA
constexpr size_t kFieldBytes = size_t(kMaxCells) * sizeof(double);
constexpr size_t kYOffset = 0;                           // Y[2][3]: stage inputs
constexpr size_t kZxOffset = kYOffset + 6 * kFieldBytes;  // bed slopes dz/dx, dz/dy
constexpr size_t kZyOffset = kZxOffset + kFieldBytes;
constexpr size_t kPartOffset = kZyOffset + kFieldBytes;
constexpr size_t kPartBytes = size_t(3 + 3 * 4) * size_t(kMaxBlocks) * sizeof(double);
constexpr size_t kCtlOffset = kPartOffset + kPartBytes;
constexpr size_t kFcOffset = kCtlOffset + 256;
constexpr size_t kScratchBytes = kFcOffset + 256;
static_assert(sizeof(svk::Ctl) <= 256 && sizeof(svk::DevForcing) <= 256, "scratch slots too small");

// The working memory. Host code must not use this name as a device address: it is only a
// host-side stand-in for the symbol. The device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_sv_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};

// Device address of g_sv_scratch on the current device. Outside stream capture it is looked
// up again on every call (cheap once the module is loaded), so a device reset or another
// context made current never leaves a stale address behind; during capture the address of the
// last uncaptured call on this device is used, so that first call must come before capture.
int scratch_address(int dev, cudaStream_t s, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) {
    svh::set_global_error("sv_timestep_noalloc: device index out of range");
    return SV_E_ARG;
  }
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) {
    svh::set_global_error(std::string("sv_timestep_noalloc: cudaStreamIsCapturing failed: ") +
                          cudaGetErrorString(e));
    return SV_E_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_sv_scratch);
    if (e != cudaSuccess || p == nullptr) {
      svh::set_global_error(std::string("sv_timestep_noalloc: cudaGetSymbolAddress failed: ") +
                            cudaGetErrorString(e));
      return SV_E_CUDA;
    }
    g_addr[dev] = static_cast<unsigned char*>(p);
  } else if (!g_addr[dev]) {
    svh::set_global_error("sv_timestep_noalloc: the first call on a device must come before stream capture");
    return SV_E_STATE;
  }
  *out = g_addr[dev];
  return SV_OK;
}

// Whether the byte ranges [a, a + n) and [b, b + n) share a byte.
bool overlap(const void* a, const void* b, size_t n) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + n && y < x + n;
}

// Controller and forcing slots are rewritten on every call (the array keeps the previous
// call's contents); the stage buffers and partial sums are fully written before being read.
__global__ void noalloc_init_kernel(svk::Ctl* ctl, svk::DevForcing* fc, double t_local, double dt,
                                    svk::DevForcing f) {
  svk::Ctl c{};
  c.t_local = t_local;
  c.dt = dt;
  *ctl = c;
  *fc = f;
}

__global__ void noalloc_result_kernel(const svk::Ctl* ctl, double* result) {
  result[0] = ctl->cn;
  result[1] = ctl->new_dt;
  result[2] = double(ctl->repeat);
}

int fail(int code, const char* msg) {
  svh::set_global_error(std::string("sv_timestep_noalloc: ") + msg);
  return code;
}

}  // namespace

extern "C" int sv_timestep_noalloc(const sv_mesh_desc* mesh, const sv_params* params, const double manning[4],
                                   const sv_forcing* forcing, const double* z, const double* h, const double* u,
                                   const double* v, double* h_out, double* u_out, double* v_out, double t_local,
                                   double dt, double* result, void* stream) {
  if (!mesh || !params || !manning || !forcing || !z || !h || !u || !v || !h_out || !u_out || !v_out || !result)
    return fail(SV_E_ARG, "null argument");
  if (params->precision != SV_F64) return fail(SV_E_ARG, "only the FP64 path is available without allocation");
  svt::Tableau tab;
  svt::StageCoefs k;
  if (!svt::named_tableau(params->rk_method, tab) || !svt::is_diagonal(tab) || !svt::stage_coefs(tab, k))
    return fail(SV_E_ARG, "the Runge-Kutta tableau must be one whose stages use only the previous stage "
                          "(euler, midpoint, heun2, ralston2, heun3, ralston3, classic)");
  if (mesh->nx == 0 || mesh->ny == 0) return fail(SV_E_ARG, "empty mesh");
  if (mesh->nx > (uint64_t)kMaxCells || mesh->ny > (uint64_t)kMaxCells ||
      (long long)(mesh->nx * mesh->ny) > kMaxCells)
    return fail(SV_E_LIMIT, "mesh larger than the 65536-cell (256 x 256) working array");
  const double dx = mesh->dx < 0 ? -mesh->dx : mesh->dx, dy = mesh->dy < 0 ? -mesh->dy : mesh->dy;
  if (!(dx > 1e-6) || !(dy > 1e-6)) return fail(SV_E_ARG, "cell size must exceed 1e-6");
  if (!(params->step_duration > 0.0)) return fail(SV_E_ARG, "step duration must be positive");
  if (forcing->rain_kind != SV_RAIN_NONE && forcing->rain_kind != SV_RAIN_UNIFORM)
    return fail(SV_E_ARG, "only uniform rain (or none) is available without allocation");
  if (forcing->head_kind != SV_HEAD_NONE && forcing->head_kind != SV_HEAD_EDGES)
    return fail(SV_E_ARG, "only edge-strip head boundaries (or none) are available without allocation");
  const long long nblk = svk::variant_partials(kVariant, (long long)mesh->nx, (long long)mesh->ny);
  if (nblk > kMaxBlocks) return fail(SV_E_LIMIT, "mesh needs more partial-sum slots than the working array holds");
  const size_t field_bytes = size_t(mesh->nx * mesh->ny) * sizeof(double);
  const double* outs[3] = {h_out, u_out, v_out};
  const double* ins[4] = {z, h, u, v};
  for (int a = 0; a < 3; ++a) {
    for (const double* i : ins)
      if (overlap(outs[a], i, field_bytes)) return fail(SV_E_ARG, "output buffers must not overlap the inputs");
    for (int b = a + 1; b < 3; ++b)
      if (overlap(outs[a], outs[b], field_bytes)) return fail(SV_E_ARG, "output buffers must not overlap each other");
  }

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SV_E_CUDA, cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* base = nullptr;
  int r = scratch_address(dev, s, &base);
  if (r != SV_OK) return r;
  double* Y = reinterpret_cast<double*>(base + kYOffset);
  double* zx = reinterpret_cast<double*>(base + kZxOffset);
  double* zy = reinterpret_cast<double*>(base + kZyOffset);
  double* part = reinterpret_cast<double*>(base + kPartOffset);
  svk::Ctl* ctl = reinterpret_cast<svk::Ctl*>(base + kCtlOffset);
  svk::DevForcing* fc = reinterpret_cast<svk::DevForcing*>(base + kFcOffset);

  svk::DevForcing f{};
  f.rain_kind = forcing->rain_kind;
  f.head_kind = forcing->head_kind;
  f.head_edges = forcing->head_edges;
  f.rq0 = forcing->rain_q0; f.rq1 = forcing->rain_q1;
  f.hh0 = forcing->head_h0; f.hh1 = forcing->head_h1;
  noalloc_init_kernel<<<1, 1, 0, s>>>(ctl, fc, t_local, dt, f);
  e = svk::launch_bed_slopes<double>(z, int(mesh->nx), int(mesh->ny), dx, dy, zx, zy, s);
  if (e != cudaSuccess) return fail(SV_E_CUDA, cudaGetErrorString(e));

  svk::StageParams<double> P{};
  P.nx = int(mesh->nx); P.ny = int(mesh->ny);
  P.dx = dx; P.dy = dy; P.L = params->step_duration;
  P.cell_area = dx * dy;
  // U_[0] is read from the inputs (cur = 0); the accumulator and U_[N] go to the outputs
  P.S[0][0] = const_cast<double*>(h); P.S[0][1] = const_cast<double*>(u); P.S[0][2] = const_cast<double*>(v);
  P.S[1][0] = h_out; P.S[1][1] = u_out; P.S[1][2] = v_out;
  P.z = z; P.zx = zx; P.zy = zy;
  for (int i = 0; i < 4; ++i) { P.man_p[i] = nullptr; P.man_s[i] = manning[i]; }
  P.fc = fc;
  P.manning = params->manning; P.rain_mode = params->rain_mode; P.head_first = params->head_first;
  P.nstages = k.N;
  P.ctl = ctl;
  P.part = part;
  P.nblk = nblk;
  const bool tally = !(params->flags & SV_FLAG_NO_TALLIES);
  for (int st = 0; st < k.N; ++st) {
    P.stage = st;
    P.c_s = k.c[st];
    P.mode = svk::M_ACC | (st == 0 ? svk::M_FIRST : 0) | (st == k.N - 1 ? svk::M_LAST : 0) | (tally ? svk::M_TALLY : 0);
    for (int j = 0; j < 4; ++j) { P.a_next[j] = k.a_next[st][j]; P.b[j] = k.b[j]; }
    const int in = (st - 1) & 1, out = st & 1;
    for (int fld = 0; fld < 3; ++fld) {
      P.Yin[fld] = st > 0 ? Y + (size_t(in) * 3 + fld) * size_t(kMaxCells) : nullptr;
      P.Yout[fld] = st < k.N - 1 ? Y + (size_t(out) * 3 + fld) * size_t(kMaxCells) : nullptr;
      P.Kout[fld] = nullptr;
      for (int j = 0; j < 4; ++j) P.Kin[j][fld] = nullptr;
    }
    e = svk::launch_variant<double>(P, kVariant, s);
    if (e != cudaSuccess) return fail(SV_E_CUDA, cudaGetErrorString(e));
  }
  svk::FinalizeParams F{};
  F.ctl = ctl;
  F.part = part;
  F.nblk = nblk;
  F.nstages = k.N;
  for (int j = 0; j < 4; ++j) F.b[j] = k.b[j];
  F.cn_target = params->cn_target;
  F.max_dt = params->max_dt;
  F.L = params->step_duration;
  F.cell_area = dx * dy;
  F.auto_mode = 0;
  F.tally = tally ? 1 : 0;
  F.is_float = 0;
  e = svk::launch_finalize(F, s);
  if (e != cudaSuccess) return fail(SV_E_CUDA, cudaGetErrorString(e));
  noalloc_result_kernel<<<1, 1, 0, s>>>(ctl, result);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(SV_E_CUDA, cudaGetErrorString(e));
  return SV_OK;
}
