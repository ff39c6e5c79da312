// sv_capi.cu -- the C-ABI of include/sv.h: device-memory owner, stage schedule and the
// graph-captured step loop. Host code only; kernels live in sv_f64.cu / sv_f32.cu.
//
// Memory layout in HBM (per solver, SoA, row-major i = y*nx + x, value type T):
//   S[2][h,u,v]  two state buffers; S[cur] holds U_[0], S[cur^1] is the RK accumulator and
//                receives U_[N]; accepting a timestep flips `cur` (no copy)
//   Y[2][h,u,v]  ping-pong stage inputs Y_1..Y_{N-1}
//   z            bed elevation (its slopes are recomputed in-kernel from the tile)
//   K[s][h,u,v]  stored stage derivatives, only for non-diagonal tableaux
//   optional per-cell Manning n / depths, rain q0/q1 or pattern, head targets
//   ctl, forcing  small device structs (controller state, per-step boundary values)
//   part         per-CTA FP64 partials of the CFL max/min, volume and tallies
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sv.h"
#include "sv_launch.h"
#include "sv_tableau.h"

using svk::Ctl;
using svk::DevForcing;

// NVTX range over one host call (a profiler shows the library's steps, advances and tuning on
// its timeline; without a tool attached a range costs a few nanoseconds)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

namespace {

thread_local std::string g_create_err;

using svt::Tableau;
using svt::named_tableau;
using svt::is_diagonal;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

namespace svh {
// error message of context-free entry points, read back by sv_last_error(NULL)
void set_global_error(const std::string& msg) { g_create_err = msg; }
}  // namespace svh

struct sv_ctx {
  virtual ~sv_ctx() {}
  std::string err;
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* where) {
    err = std::string(where) + ": " + cudaGetErrorString(e);
    return SV_E_CUDA;
  }
  virtual int set_field(int id, const double* host, uint64_t n) = 0;
  virtual int get_field(int id, double* host, uint64_t n) = 0;
  virtual int set_manning(double, double, double, double) = 0;
  virtual int set_eddy(int, double, double, double) = 0;
  virtual int set_source_order(const int*, int) = 0;
  virtual int set_forcing(const sv_forcing*) = 0;
  virtual int set_dt(double) = 0;
  virtual int get_dt(double*) = 0;
  virtual int eval_dudt(int, double, double) = 0;
  virtual int do_timestep(double, double, double*, int*, double*) = 0;
  virtual int accept() = 0;
  virtual int advance(sv_stats*) = 0;
  virtual int get_stats(sv_stats*) = 0;
  virtual int set_stats(const sv_stats*) = 0;
  virtual int run_timesteps(uint64_t, int, sv_stats*, int*, sv_timing*) = 0;
  virtual int set_variant(int) = 0;
  virtual int get_variant() const = 0;
  virtual int autotune(int*) = 0;
  virtual float autotune_ms(int v) const = 0;
  double last_advance_ms = -1.0;
};

namespace {

// FP64 staging buffers of field transfers come from one stream-ordered pool per device that
// keeps freed memory mapped. The device's default pool unmaps freed memory at every
// synchronisation, and mapping it again costs more than the copy itself (5-20 ms against
// 2.5 ms for a 134 MB field). Destroying a solver trims the pool back to nothing.
cudaMemPool_t staging_pool(int device, bool create) {
  static std::mutex mu;
  static std::map<int, cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  auto it = pools.find(device);
  if (it != pools.end()) return it->second;
  if (!create) return nullptr;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;  // the caller falls back to the default pool
  }
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools[device] = pool;
  return pool;
}

#define SV_CUDA(call)                                  \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

template <typename T>
struct Solver final : public sv_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  sv_mesh_desc mesh{};
  sv_params prm{};
  Tableau tab;
  bool diag = true;
  int N = 4;
  int tile = 0;      // tile shape of the volume kernel
  int variant = 5;   // stage-kernel variant (svk::launch_variant)
  float tune_ms[svk::kNumVariants] = {};
  float autotune_ms(int v) const override { return v >= 0 && v < svk::kNumVariants ? tune_ms[v] : 0.0f; }
  int tx = 32, ty = 8;
  long long ncells = 0, nfaces = 0, nblk = 0, vol_nblk = 0;
  T* S[2][3] = {};
  T* Y[2][3] = {};
  T* K[4][3] = {};
  T* z = nullptr;                  // bed (FP32-with-datum mode: offset from the tile datum)
  T *zx = nullptr, *zy = nullptr;  // bed slopes (Constants.cpp:39-40)
  bool datum = false;              // SV_F32_DATUM64
  double* zdat = nullptr;          // per datum tile FP64 datum
  int dtiles_x = 0, dtiles_y = 0;
  T* man[4] = {};
  double man_s[4] = {0.03, 0.3, 0.1, 0.3};  // ManningRoughnessSourceTerm.cpp:99-102
  int* d_flag = nullptr;  // result of a field comparison on the device
  T *q0 = nullptr, *q1 = nullptr, *pat = nullptr, *hb0 = nullptr, *hb1 = nullptr;
  T *irate = nullptr, *icap = nullptr;  // InfiltrationSourceTerm fields (.hpp:106-109)
  T *efx = nullptr, *efy = nullptr;     // EnergyLossSourceTerm fields (.hpp:199-202)
  T* hcomp[2] = {};                     // FP32: compensation of the depth update, per state parity
  // EddyViscositySourceTerm (EddyViscositySourceTerm.cpp:112-137): mode (SV_EDDY_*), the
  // constant coefficient ("default mu", or the per-cell field) and the Smagorinsky
  // coefficients ("constant coefficient", "dynamic coefficient")
  int eddy_mode = SV_EDDY_OFF;
  double eddy_mu = 1.0, eddy_c = 0.05, eddy_s = 0.5;
  T* eddy_mup = nullptr;
  int term_order_[3] = {SV_TERM_MANNING, SV_TERM_ELOSS, SV_TERM_EDDY};
  bool order_set = false;  // else roughness / energy loss per SV_FLAG_ELOSS_FIRST, then eddy viscosity
  // FP32 with the batches' variant runs the batched column sweep as a batch of one, so a
  // solver on its own and a batch member execute the same machine code and give the same
  // bits (FP32 is contracted per kernel); that kernel reads its parameters from device memory
  svk::StageParams<T>* d_sp = nullptr;  // [N] stage parameters + [1] for the autotuner
  long long* d_ws = nullptr;            // warp starts: {0, nblk} and, for the autotuner, {0, n}
  unsigned long long sp_version = ~0ull;
  // debug buffers (per-function parity path)
  T* dbg_slp[8] = {};
  T* dbg_face[5] = {};
  T *dbg_nh = nullptr, *dbg_sf = nullptr;
  T* dbg_k[3] = {};
  Ctl* ctl = nullptr;
  Ctl* dbg_ctl = nullptr;
  DevForcing* fc = nullptr;
  double* part = nullptr;
  double* scalar = nullptr;
  int cur = 0;  // host mirror of ctl->cur
  cudaGraphExec_t graph = nullptr;
  bool graph_dirty = true;
  unsigned long long pversion = 0;  // bumped whenever launch parameters change
  int unroll = 8;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<void*> owned;
  T* n_deep_own = nullptr;  // n_deep's own array once it differs from n_shallow
  T* pslp[6] = {};          // split schedule: slopes of the stage input (allocated on first use)
  int ensure_split() {
    if (pslp[0]) return SV_OK;
    for (int f = 0; f < 6; ++f) SV_CUDA(alloc_cells(&pslp[f], false));
    graph_dirty = true; ++pversion;
    return SV_OK;
  }
  // interior / general strip lists of the column sweep, per strip height (16, 32, 64 rows):
  // interior strips (whole window inside the mesh, no coded-out bed) run the interior kernel
  struct Strips {
    int* d_i = nullptr;
    int* d_b = nullptr;
    int ni = 0, nb = 0;
    // two-cells-per-lane variants (FP32): pairs of adjacent interior strips (first strip of
    // each, nx even) and the interior strips left out of a pair
    int* d_p = nullptr;
    int* d_pi = nullptr;
    int np = 0, npi = 0;
    bool valid = false;
  };
  Strips strips_[3];
  unsigned char* d_sflags = nullptr;
  static int strips_slot(int rows) { return rows == 16 ? 0 : (rows == 32 ? 1 : 2); }
  void invalidate_strips() {
    for (Strips& x : strips_) x.valid = false;
    graph_dirty = true; ++pversion;
  }
  // the lists for variant v (a column-sweep variant), built from the bed on the device
  int ensure_strips(int v) {
    const int rows = svk::variant_sweep_rows(v);
    if (rows == 0) return SV_OK;
    Strips& L = strips_[strips_slot(rows)];
    if (L.valid) return SV_OK;
    const long long n = svk::variant_partials(v, (long long)mesh.nx, (long long)mesh.ny);
    if (!L.d_i) {
      SV_CUDA(alloc(&L.d_i, size_t(n)));
      SV_CUDA(alloc(&L.d_b, size_t(n)));
      SV_CUDA(alloc(&L.d_p, size_t(n)));
      SV_CUDA(alloc(&L.d_pi, size_t(n)));
    }
    if (!d_sflags)  // sized for the shortest strips, which are the most numerous
      SV_CUDA(alloc(&d_sflags, size_t(svk::variant_partials(4, (long long)mesh.nx, (long long)mesh.ny))));
    cudaError_t e = svk::launch_strip_flags<T>(z, int(mesh.nx), int(mesh.ny), rows, n, d_sflags, stream);
    if (e != cudaSuccess) return cuda_fail(e, "strip flags");
    std::vector<unsigned char> flags(static_cast<size_t>(n));
    SV_CUDA(cudaMemcpyAsync(flags.data(), d_sflags, size_t(n), cudaMemcpyDeviceToHost, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    std::vector<int> in, bd, pr, pin;
    for (long long i = 0; i < n; ++i) (flags[size_t(i)] ? in : bd).push_back(int(i));
    // pairs: strips (2t, 2t+1) of one row band, both interior; their vector loads need an even
    // row length (every row then starts 8-byte aligned)
    const long long tiles_x = (static_cast<long long>(mesh.nx) + svk::kSweepOut - 1) / svk::kSweepOut;
    for (long long i = 0; i < n; ++i) {
      if (!flags[size_t(i)]) continue;
      const long long tx = i % tiles_x;
      if (mesh.nx % 2 == 0 && tx % 2 == 0 && tx + 1 < tiles_x && flags[size_t(i + 1)]) {
        pr.push_back(int(i));
        ++i;  // the pair's second strip
      } else {
        pin.push_back(int(i));
      }
    }
    auto up = [&](int* d, const std::vector<int>& h) -> cudaError_t {
      if (h.empty()) return cudaSuccess;
      return cudaMemcpyAsync(d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, stream);
    };
    SV_CUDA(up(L.d_i, in));
    SV_CUDA(up(L.d_b, bd));
    SV_CUDA(up(L.d_p, pr));
    SV_CUDA(up(L.d_pi, pin));
    SV_CUDA(cudaStreamSynchronize(stream));
    L.ni = int(in.size());
    L.nb = int(bd.size());
    L.np = int(pr.size());
    L.npi = int(pin.size());
    L.valid = true;
    graph_dirty = true; ++pversion;
    return SV_OK;
  }
  // the strip lists of variant v into P (none for other variants or lists not built yet)
  void set_strips(svk::StageParams<T>& P, int v) const {
    const int rows = svk::variant_sweep_rows(v);
    P.istrips = P.bstrips = nullptr;
    P.ipairs = nullptr;
    P.n_istrips = P.n_bstrips = P.n_ipairs = 0;
    if (rows == 0) return;
    const Strips& L = strips_[strips_slot(rows)];
    if (!L.valid) return;
    P.bstrips = L.d_b; P.n_bstrips = L.nb;
    if (svk::variant_is_pair(v)) {
      P.ipairs = L.d_p; P.n_ipairs = L.np;
      P.istrips = L.d_pi; P.n_istrips = L.npi;
    } else {
      P.istrips = L.d_i; P.n_istrips = L.ni;
    }
  }

  ~Solver() override {
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    for (void* p : owned) cudaFree(p);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
    if (cudaMemPool_t pool = staging_pool(device, false)) cudaMemPoolTrimTo(pool, 0);
  }

  size_t device_bytes = 0;
  template <typename U> cudaError_t alloc(U** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = count * sizeof(U) > 0 ? count * sizeof(U) : 16;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return e;
    device_bytes += bytes;
    owned.push_back(q);
    *p = static_cast<U*>(q);
    return cudaSuccess;
  }
  cudaError_t alloc_cells(T** p, bool zero = true) {
    cudaError_t e = alloc(p, size_t(ncells));
    if (e == cudaSuccess && zero) e = cudaMemsetAsync(*p, 0, size_t(ncells) * sizeof(T), stream);
    return e;
  }

  int init(const sv_mesh_desc* m, const sv_params* p, int dev) {
    mesh = *m;
    prm = *p;
    device = dev;
    if (!named_tableau(p->rk_method, tab)) return fail(SV_E_ARG, "unknown Runge Kutta scheme index");
    N = tab.nsteps();
    diag = is_diagonal(tab);
    if (m->nx == 0 || m->ny == 0) return fail(SV_E_ARG, "empty mesh");
    if (m->nx > 0x7fffffffull || m->ny > 0x7fffffffull) return fail(SV_E_LIMIT, "mesh side above 2^31-1");
    if (!(std::fabs(m->dx) > 1e-6) || !(std::fabs(m->dy) > 1e-6)) return fail(SV_E_ARG, "cell size must exceed 1e-6");
    if (!(p->step_duration > 0.0)) return fail(SV_E_ARG, "step duration must be positive");
    mesh.dx = std::fabs(m->dx);
    mesh.dy = std::fabs(m->dy);
    ncells = (long long)m->nx * (long long)m->ny;
    nfaces = (long long)(m->nx + 1) * (long long)m->ny + (long long)(m->ny + 1) * (long long)m->nx;
    tx = svk::kTiles[tile].tx;
    ty = svk::kTiles[tile].ty;
    nblk = svk::variant_partials(variant, (long long)m->nx, (long long)m->ny);
    vol_nblk = (long long)((m->nx + tx - 1) / tx) * (long long)((m->ny + ty - 1) / ty);
    SV_CUDA(cudaSetDevice(dev));
    SV_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SV_CUDA(cudaEventCreate(&ev0));
    SV_CUDA(cudaEventCreate(&ev1));
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 3; ++f) {
        SV_CUDA(alloc_cells(&S[b][f]));
        SV_CUDA(alloc_cells(&Y[b][f], false));
      }
    if (!diag)
      for (int s = 0; s < N - 1; ++s)
        for (int f = 0; f < 3; ++f) SV_CUDA(alloc_cells(&K[s][f], false));
    SV_CUDA(alloc_cells(&z));
    SV_CUDA(alloc_cells(&zx));
    SV_CUDA(alloc_cells(&zy));
    if (sizeof(T) == 4) {  // zero compensation: a new state carries none
      SV_CUDA(alloc_cells(&hcomp[0]));
      SV_CUDA(alloc_cells(&hcomp[1]));
    }
    datum = (p->precision == SV_F32_DATUM64);
    if (datum) {
      dtiles_x = int((m->nx + svk::kDatumTX - 1) / svk::kDatumTX);
      dtiles_y = int((m->ny + svk::kDatumTY - 1) / svk::kDatumTY);
      SV_CUDA(alloc(&zdat, size_t(dtiles_x) * dtiles_y));
      SV_CUDA(cudaMemsetAsync(zdat, 0, sizeof(double) * size_t(dtiles_x) * dtiles_y, stream));
    }
    SV_CUDA(alloc(&ctl, 1));
    SV_CUDA(alloc(&dbg_ctl, 1));
    SV_CUDA(alloc(&fc, 1));
    long long maxp = vol_nblk;
    for (int v = 0; v < svk::kNumVariants; ++v) maxp = std::max(maxp, svk::variant_partials(v, m->nx, m->ny));
    SV_CUDA(alloc(&part, size_t(svk::part_count(maxp, N))));
    SV_CUDA(alloc(&scalar, 4));
    Ctl c{};
    c.dt = p->initial_dt;
    SV_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaMemcpyAsync(dbg_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    DevForcing f{};
    SV_CUDA(cudaMemcpyAsync(fc, &f, sizeof(DevForcing), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }

  T** field_slot(int id, bool& lazy) {
    lazy = false;
    switch (id) {
      case SV_FIELD_Z: return &z;
      case SV_FIELD_H: return &S[cur][0];
      case SV_FIELD_U: return &S[cur][1];
      case SV_FIELD_V: return &S[cur][2];
      case SV_FIELD_N_SHALLOW: lazy = true; return &man[0];
      case SV_FIELD_N_DEEP: lazy = true; return &man[1];
      case SV_FIELD_D_SHALLOW: lazy = true; return &man[2];
      case SV_FIELD_D_DEEP: lazy = true; return &man[3];
      case SV_FIELD_QBDY0: lazy = true; return &q0;
      case SV_FIELD_QBDY1: lazy = true; return &q1;
      case SV_FIELD_HBDY0: lazy = true; return &hb0;
      case SV_FIELD_HBDY1: lazy = true; return &hb1;
      case SV_FIELD_RAIN_PATTERN: lazy = true; return &pat;
      case SV_FIELD_INFIL_RATE: lazy = true; return &irate;
      case SV_FIELD_INFIL_CAP: lazy = true; return &icap;
      case SV_FIELD_ELOSS_FX: lazy = true; return &efx;
      case SV_FIELD_ELOSS_FY: lazy = true; return &efy;
      case SV_FIELD_H_COMP: return hcomp[cur] ? &hcomp[cur] : nullptr;
      case SV_FIELD_EDDY_MU: lazy = true; return &eddy_mup;
    }
    return nullptr;
  }

  // Fields cross the interface in FP64. An FP64 solver copies them straight between the host
  // buffer and its own array; another value type stages them in a stream-ordered FP64
  // buffer and converts on the device, so a field costs one copy at the link's speed (DMA
  // when the caller's buffer is pinned) and no pass over it on the host.
  cudaError_t stage_alloc(double** p, uint64_t n) {
    const size_t bytes = std::max<uint64_t>(n, 1) * sizeof(double);
    cudaMemPool_t pool = staging_pool(device, true);
    return pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, stream)
                : cudaMallocAsync(reinterpret_cast<void**>(p), bytes, stream);
  }
  int upload(T* dst, const double* host, uint64_t n) {
    cudaError_t e;
    if constexpr (std::is_same<T, double>::value) {
      e = cudaMemcpyAsync(dst, host, n * sizeof(double), cudaMemcpyHostToDevice, stream);
    } else {
      double* st = nullptr;
      SV_CUDA(stage_alloc(&st, n));
      e = cudaMemcpyAsync(st, host, n * sizeof(double), cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess) e = svk::launch_from_f64<T>(st, dst, (long long)n, stream);
      cudaError_t f = cudaFreeAsync(st, stream);
      if (e == cudaSuccess) e = f;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "field upload");
    return SV_OK;
  }
  int download(const T* src, double* host, uint64_t n, bool absolute_bed = false) {
    cudaError_t e;
    if constexpr (std::is_same<T, double>::value) {
      (void)absolute_bed;
      e = cudaMemcpyAsync(host, src, n * sizeof(double), cudaMemcpyDeviceToHost, stream);
    } else {
      double* st = nullptr;
      SV_CUDA(stage_alloc(&st, n));
      if (absolute_bed)  // FP32 with tile datums: bed = FP64 datum + FP32 offset
        e = svk::launch_datum_absolute(reinterpret_cast<const float*>(src), int(mesh.nx), int(mesh.ny), dtiles_x, zdat,
                                       st, stream);
      else
        e = svk::launch_to_f64<T>(src, st, (long long)n, stream);
      if (e == cudaSuccess) e = cudaMemcpyAsync(host, st, n * sizeof(double), cudaMemcpyDeviceToHost, stream);
      cudaError_t f = cudaFreeAsync(st, stream);
      if (e == cudaSuccess) e = f;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "field download");
    return SV_OK;
  }

  int set_field(int id, const double* host, uint64_t n) override {
    if (!host) return fail(SV_E_ARG, "null host pointer");
    if ((long long)n != ncells) return fail(SV_E_ARG, "field size mismatch");
    bool lazy;
    T** slot = field_slot(id, lazy);
    if (!slot) return fail(SV_E_ARG, "field id not settable");
    if (id == SV_FIELD_N_DEEP && man[0]) return set_n_deep(host, n);
    if (id == SV_FIELD_N_SHALLOW && man[1] && man[1] == man[0]) {
      // n_deep shares n_shallow's array: it keeps its values in an array of its own (one per
      // solver, reused whenever the two part again)
      if (!n_deep_own) SV_CUDA(alloc_cells(&n_deep_own, false));
      SV_CUDA(cudaMemcpyAsync(n_deep_own, man[0], size_t(ncells) * sizeof(T), cudaMemcpyDeviceToDevice, stream));
      man[1] = n_deep_own;
      graph_dirty = true; ++pversion;
    }
    if (lazy && *slot == nullptr) {
      SV_CUDA(alloc_cells(slot, false));
      graph_dirty = true; ++pversion;
    }
    if (id == SV_FIELD_Z && datum) return set_bed_with_datum(host, n);
    int r = upload(*slot, host, n);
    if (r == SV_OK && id == SV_FIELD_H && hcomp[0]) {  // a new depth field carries no compensation
      SV_CUDA(cudaMemsetAsync(hcomp[0], 0, size_t(ncells) * sizeof(T), stream));
      SV_CUDA(cudaMemsetAsync(hcomp[1], 0, size_t(ncells) * sizeof(T), stream));
      SV_CUDA(cudaStreamSynchronize(stream));
    }
    if (r == SV_OK && id == SV_FIELD_Z) {
      cudaError_t e = svk::launch_bed_slopes<T>(z, int(mesh.nx), int(mesh.ny), mesh.dx, mesh.dy, zx, zy, stream);
      if (e != cudaSuccess) return cuda_fail(e, "bed slopes");
      SV_CUDA(cudaStreamSynchronize(stream));
      invalidate_strips();
    }
    return r;
  }

  // n_deep equal to n_shallow once both are in the solver's value type (compared bit for bit
  // on the device): the kernels read one array. Otherwise n_deep gets an array of its own.
  int set_n_deep(const double* host, uint64_t n) {
    double* st = nullptr;
    if (!d_flag) SV_CUDA(alloc(&d_flag, 1));
    SV_CUDA(stage_alloc(&st, n));
    int flag = 0;
    cudaError_t e = cudaMemcpyAsync(st, host, n * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_flag, 0, sizeof(int), stream);
    if (e == cudaSuccess) e = svk::launch_differs<T>(st, man[0], (long long)n, d_flag, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && flag) {
      if (!man[1] || man[1] == man[0]) {
        if (!n_deep_own) e = alloc_cells(&n_deep_own, false);
        man[1] = n_deep_own;
        graph_dirty = true; ++pversion;
      }
      if (e == cudaSuccess) e = svk::launch_from_f64<T>(st, man[1], (long long)n, stream);
    } else if (e == cudaSuccess && man[1] != man[0]) {
      man[1] = man[0];
      graph_dirty = true; ++pversion;
    }
    cudaError_t f = cudaFreeAsync(st, stream);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "n_deep upload");
    return SV_OK;
  }

  // FP32-with-datum bed: per 32 x 8 tile datum = the tile's lowest bed rounded down to a
  // multiple of 2^-10 m (datum differences are then exact in FP64); stored bed = FP32
  // offset from it; bed slopes from the FP64 bed (Minmod3 in FP64, rounded once).
  int set_bed_with_datum(const double* host, uint64_t n) {
    if constexpr (!std::is_same<T, float>::value) {
      (void)host; (void)n;
      return fail(SV_E_STATE, "tile datums need an FP32 solver");
    } else {
      invalidate_strips();
      double* dz = nullptr;
      SV_CUDA(stage_alloc(&dz, n));
      cudaError_t e = cudaMemcpyAsync(dz, host, n * sizeof(double), cudaMemcpyHostToDevice, stream);
      if (e == cudaSuccess)
        e = svk::launch_datum_bed(dz, int(mesh.nx), int(mesh.ny), mesh.dx, mesh.dy, dtiles_x, dtiles_y, zdat, z, zx, zy,
                                  stream);
      cudaError_t f = cudaFreeAsync(dz, stream);
      if (e == cudaSuccess) e = f;
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return cuda_fail(e, "datum bed");
      return SV_OK;
    }
  }

  int debug_ptr(int id, T*& p, long long& count) {
    count = ncells;
    p = nullptr;
    if (id >= SV_FIELD_DHDX && id <= SV_FIELD_DZDY) {
      static const int map[8] = {0, 1, 2, 4, 5, 6, 3, 7};  // DHDX,DUDX,DVDX,DHDY,DUDY,DVDY,DZDX,DZDY
      p = dbg_slp[map[id - SV_FIELD_DHDX]];
    } else if (id >= SV_FIELD_FLUX_H && id <= SV_FIELD_FLUX_BRANCH) {
      p = dbg_face[id - SV_FIELD_FLUX_H];
      count = nfaces;
    } else if (id >= SV_FIELD_DHDT && id <= SV_FIELD_DVDT) {
      p = dbg_k[id - SV_FIELD_DHDT];
    }
    return p ? SV_OK : fail(SV_E_STATE, "field not available: run sv_eval_dudt first");
  }

  int get_field(int id, double* host, uint64_t n) override {
    if (!host) return fail(SV_E_ARG, "null host pointer");
    const T* src = nullptr;
    long long count = ncells;
    bool lazy;
    if (id >= SV_FIELD_STATE_BASE && id < SV_FIELD_STATE_BASE + 3 * (N + 1)) {
      int s = (id - SV_FIELD_STATE_BASE) / 3, f = (id - SV_FIELD_STATE_BASE) % 3;
      if (s == 0) src = S[cur][f];
      else if (s == N) src = S[cur ^ 1][f];
      else return fail(SV_E_ARG, "intermediate stage states are not stored");
    } else if (id >= SV_FIELD_K_BASE && id < SV_FIELD_K_BASE + 3 * N) {
      int s = (id - SV_FIELD_K_BASE) / 3, f = (id - SV_FIELD_K_BASE) % 3;
      if (s == 0 && dbg_k[f]) src = dbg_k[f];
      else if (!diag && s < N - 1) src = K[s][f];
      else return fail(SV_E_ARG, "stage derivative not stored");
    } else if (id >= 20) {
      T* p;
      int r = debug_ptr(id, p, count);
      if (r) return r;
      src = p;
    } else {
      T** slot = field_slot(id, lazy);
      if (!slot) return fail(SV_E_ARG, "unknown field id");
      if (!*slot) return fail(SV_E_STATE, "field was never set");
      src = *slot;
    }
    if ((long long)n != count) return fail(SV_E_ARG, "field size mismatch");
    return download(src, host, n, datum && id == SV_FIELD_Z);
  }

  int term_order() const {
    int t[3] = {term_order_[0], term_order_[1], term_order_[2]};
    if (!order_set && (prm.flags & SV_FLAG_ELOSS_FIRST)) { t[0] = SV_TERM_ELOSS; t[1] = SV_TERM_MANNING; }
    return t[0] | (t[1] << 2) | (t[2] << 4);
  }
  int set_eddy(int mode, double mu, double mc, double ms) override {
    if (mode < SV_EDDY_OFF || mode > SV_EDDY_SMAGORINSKY) return fail(SV_E_ARG, "unknown eddy viscosity mode");
    if (!std::isfinite(mu) || !std::isfinite(mc) || !std::isfinite(ms))
      return fail(SV_E_ARG, "eddy viscosity coefficients must be finite");
    eddy_mode = mode; eddy_mu = mu; eddy_c = mc; eddy_s = ms;
    graph_dirty = true; ++pversion;
    return SV_OK;
  }
  int set_source_order(const int* terms, int n) override {
    if (n < 0 || n > 3 || (n > 0 && !terms)) return fail(SV_E_ARG, "at most three source terms");
    int t[3], k = 0;
    bool seen[4] = {};
    for (int i = 0; i < n; ++i) {
      if (terms[i] < SV_TERM_MANNING || terms[i] > SV_TERM_EDDY || seen[terms[i]])
        return fail(SV_E_ARG, "source order lists roughness, energy loss and eddy viscosity at most once each");
      seen[terms[i]] = true;
      t[k++] = terms[i];
    }
    for (int x = SV_TERM_MANNING; x <= SV_TERM_EDDY; ++x)
      if (!seen[x]) t[k++] = x;  // terms not listed follow in the default order
    for (int i = 0; i < 3; ++i) term_order_[i] = t[i];
    order_set = true;
    graph_dirty = true; ++pversion;
    return SV_OK;
  }
  int set_manning(double a, double b, double c, double d) override {
    man_s[0] = a; man_s[1] = b; man_s[2] = c; man_s[3] = d;
    for (int i = 0; i < 4; ++i) man[i] = nullptr;  // uniform values replace per-cell fields
    graph_dirty = true; ++pversion;
    return SV_OK;
  }

  // Checks one step's boundary values against the fields this solver holds and converts
  // them to the device form. `may_alloc`: allocate the (cleared) discharge fields that
  // SV_RAIN_FIELDS needs (BoundarySourceTerm::clear_values); a queued batch step may not.
  int make_forcing(const sv_forcing* f, DevForcing* d, bool may_alloc) {
    if (!f) return fail(SV_E_ARG, "null forcing");
    if (f->rain_kind < 0 || f->rain_kind > 3 || f->head_kind < 0 || f->head_kind > 4)
      return fail(SV_E_ARG, "bad forcing kind");
    if (f->rain_kind == SV_RAIN_FIELDS && (!q0 || !q1)) {
      if (!may_alloc) return fail(SV_E_STATE, "discharge fields not set");
      if (!q0) { SV_CUDA(alloc_cells(&q0)); graph_dirty = true; ++pversion; }
      if (!q1) { SV_CUDA(alloc_cells(&q1)); graph_dirty = true; ++pversion; }
    }
    if (f->rain_kind == SV_RAIN_PATTERN && !pat) return fail(SV_E_STATE, "rain pattern field not set");
    if ((f->head_kind == SV_HEAD_FIELDS || f->head_kind == SV_STAGE_FIELDS) && (!hb0 || !hb1))
      return fail(SV_E_STATE, "head fields not set");
    *d = DevForcing{};
    d->rain_kind = f->rain_kind;
    d->head_kind = f->head_kind;
    d->head_edges = f->head_edges;
    d->rq0 = f->rain_q0; d->rq1 = f->rain_q1;
    d->hh0 = f->head_h0; d->hh1 = f->head_h1;
    return SV_OK;
  }

  int set_forcing(const sv_forcing* f) override {
    DevForcing d;
    int r = make_forcing(f, &d, true);
    if (r) return r;
    SV_CUDA(cudaMemcpyAsync(fc, &d, sizeof(d), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }

  int read_ctl(Ctl& c) {
    SV_CUDA(cudaMemcpyAsync(&c, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    cur = c.cur;
    return SV_OK;
  }
  int write_ctl_time(double t_local, double dt) {
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    c.t_local = t_local;
    c.dt = dt;
    c.done = 0;
    SV_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }
  int set_dt(double dt) override {
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    return write_ctl_time(c.t_local, dt);
  }
  int get_dt(double* dt) override {
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    *dt = c.dt;
    return SV_OK;
  }

  svk::StageParams<T> base_params() const {
    svk::StageParams<T> P{};
    P.nx = int(mesh.nx); P.ny = int(mesh.ny);
    P.dx = mesh.dx; P.dy = mesh.dy; P.L = prm.step_duration;
    P.cell_area = mesh.dx * mesh.dy;
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 3; ++f) P.S[b][f] = S[b][f];
    P.z = z;
    P.zx = zx;
    P.zy = zy;
    P.zdat = datum ? zdat : nullptr;
    P.dtiles_x = dtiles_x;
    for (int f = 0; f < 6; ++f) P.pslp[f] = pslp[f];
    for (int i = 0; i < 4; ++i) { P.man_p[i] = man[i]; P.man_s[i] = T(man_s[i]); }
    P.fc = fc;
    P.q0p = q0; P.q1p = q1; P.pat = pat; P.hb0p = hb0; P.hb1p = hb1;
    // a source term runs once both of its fields are set (the reference builds each with
    // both fields, ...SourceTerm::create_source_term)
    P.irate = (irate && icap) ? irate : nullptr;
    P.icap = (irate && icap) ? icap : nullptr;
    P.efx = (efx && efy) ? efx : nullptr;
    P.efy = (efx && efy) ? efy : nullptr;
    P.eloss_first = (prm.flags & SV_FLAG_ELOSS_FIRST) ? 1 : 0;
    P.eddy = eddy_mode;
    P.eddy_mu = T(eddy_mu); P.eddy_c = T(eddy_c); P.eddy_s = T(eddy_s);
    P.eddy_mup = eddy_mup;
    P.term_order = term_order();
    P.hc[0] = hcomp[0];
    P.hc[1] = hcomp[1];
    P.manning = prm.manning; P.rain_mode = prm.rain_mode; P.head_first = prm.head_first;
    P.nstages = N;
    P.ctl = ctl;
    P.part = part;
    P.nblk = nblk;
    return P;
  }

  // Launch the N stages of one timestep and the finalize kernel (RungeKutta.cpp:147-167).
  // Stage s of a timestep (RungeKutta.cpp:147-153): mode, RK coefficients and buffers.
  svk::StageParams<T> stage_params(int st) const {
    svk::StageParams<T> P = base_params();
    set_strips(P, variant);
    const bool tally = !(prm.flags & SV_FLAG_NO_TALLIES);
    P.stage = st;
    P.c_s = tab.c(st + 1);
    int mode = 0;
    if (st == 0) mode |= svk::M_FIRST;
    if (st == N - 1) mode |= svk::M_LAST;
    if (diag) mode |= svk::M_ACC;
    else if (st < N - 1) mode |= svk::M_STOREK;
    if (tally) mode |= svk::M_TALLY;
    P.mode = mode;
    for (int j = 0; j < 4; ++j) { P.a_next[j] = 0.0; P.b[j] = 0.0; }
    if (st < N - 1)
      for (int j = 0; j <= st; ++j) P.a_next[j] = tab.A(st + 2, j + 1);
    for (int j = 0; j < N; ++j) P.b[j] = tab.b(j + 1);
    // stage inputs: U_[0] (s = 0), then Y[0], Y[1], Y[0] ...
    const int in = (st - 1) & 1, out = st & 1;
    for (int f = 0; f < 3; ++f) {
      P.Yin[f] = st > 0 ? Y[in][f] : nullptr;
      P.Yout[f] = st < N - 1 ? Y[out][f] : nullptr;
      P.Kout[f] = (!diag && st < N - 1) ? K[st][f] : nullptr;
      for (int j = 0; j < 4; ++j) P.Kin[j][f] = (!diag && j < N - 1) ? K[j][f] : nullptr;
    }
    return P;
  }
  svk::FinalizeParams finalize_params(bool auto_mode) const {
    svk::FinalizeParams F{};
    F.ctl = ctl;
    F.part = part;
    F.nblk = nblk;
    F.nstages = N;
    for (int j = 0; j < 4; ++j) F.b[j] = j < N ? tab.b(j + 1) : 0.0;
    F.cn_target = prm.cn_target;
    F.max_dt = prm.max_dt;
    F.L = prm.step_duration;
    F.cell_area = mesh.dx * mesh.dy;
    F.auto_mode = auto_mode ? 1 : 0;
    F.tally = (prm.flags & SV_FLAG_NO_TALLIES) ? 0 : 1;
    F.is_float = sizeof(T) == 4;
    return F;
  }

  bool batch_path(int v) const { return sizeof(T) == 4 && v == svk::batch_variant<T>(); }
  bool pow2_mesh() const {
    int e;
    return std::frexp(mesh.dx, &e) == 0.5 && std::frexp(mesh.dy, &e) == 0.5;
  }
  // Device copy of the stage parameters for the batch-of-one path (outside stream capture).
  int ensure_dev_params() {
    if (!batch_path(variant)) return ensure_strips(variant);
    if (sp_version == pversion) return SV_OK;
    if (!d_sp) {
      SV_CUDA(alloc(&d_sp, size_t(N + 1)));
      SV_CUDA(alloc(&d_ws, size_t(4)));
    }
    std::vector<svk::StageParams<T>> hp(N);
    for (int st = 0; st < N; ++st) hp[st] = stage_params(st);
    long long ws[2] = {0, nblk};
    SV_CUDA(cudaMemcpyAsync(d_sp, hp.data(), sizeof(svk::StageParams<T>) * N, cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaMemcpyAsync(d_ws, ws, sizeof(ws), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    sp_version = pversion;
    return SV_OK;
  }
  cudaError_t launch_stage_kernel(const svk::StageParams<T>& P, int st) {
    if (batch_path(variant))
      return svk::launch_sweep_batch<T>(d_sp + st, d_ws, 1, nblk, pow2_mesh(), eddy_mode != SV_EDDY_OFF, stream);
    return svk::launch_variant<T>(P, variant, stream);
  }

  // Launch the N stages of one timestep and the finalize kernel (RungeKutta.cpp:147-167).
  // ev: if non-null, 2*(N+1) events recorded around every kernel (stages, then finalize)
  int enqueue_timestep(bool auto_mode, cudaEvent_t* ev = nullptr) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    SV_CUDA(cudaStreamIsCapturing(stream, &cs));
    if (cs == cudaStreamCaptureStatusNone) {
      int r = ensure_dev_params();
      if (r) return r;
    } else if (batch_path(variant) && sp_version != pversion) {
      return fail(SV_E_STATE, "stage parameters not on the device before capture");
    }
    for (int st = 0; st < N; ++st) {
      svk::StageParams<T> P = stage_params(st);
      if (ev) SV_CUDA(cudaEventRecord(ev[2 * st], stream));
      cudaError_t e = launch_stage_kernel(P, st);
      if (e != cudaSuccess) return cuda_fail(e, "stage kernel");
      if (ev) SV_CUDA(cudaEventRecord(ev[2 * st + 1], stream));
    }
    svk::FinalizeParams F = finalize_params(auto_mode);
    if (ev) SV_CUDA(cudaEventRecord(ev[2 * N], stream));
    cudaError_t e = svk::launch_finalize(F, stream);
    if (e != cudaSuccess) return cuda_fail(e, "finalize kernel");
    if (ev) SV_CUDA(cudaEventRecord(ev[2 * N + 1], stream));
    return SV_OK;
  }

  int eval_dudt(int state_no, double t_sub, double dt) override {
    if (state_no != 0) return fail(SV_E_ARG, "only U_[0] is stored between calls");
    if (datum) return fail(SV_E_STATE, "per-function evaluation is not available with tile datums");
    if (!dbg_k[0]) {
      for (int f = 0; f < 3; ++f) SV_CUDA(alloc_cells(&dbg_k[f]));
      for (int f = 0; f < 8; ++f) SV_CUDA(alloc_cells(&dbg_slp[f]));
      for (int f = 0; f < 5; ++f) {
        SV_CUDA(alloc(&dbg_face[f], size_t(nfaces)));
        SV_CUDA(cudaMemsetAsync(dbg_face[f], 0, size_t(nfaces) * sizeof(T), stream));
      }
      SV_CUDA(alloc_cells(&dbg_nh));
      SV_CUDA(alloc_cells(&dbg_sf));
    }
    Ctl c{};
    c.t_local = t_sub;
    c.dt = dt;
    SV_CUDA(cudaMemcpyAsync(dbg_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    svk::StageParams<T> P = base_params();
    P.ctl = dbg_ctl;
    P.c_s = 0.0;
    for (int f = 0; f < 3; ++f) P.Kout[f] = dbg_k[f];
    svk::DebugParams<T> D{};
    D.nx = int(mesh.nx); D.ny = int(mesh.ny); D.dx = mesh.dx; D.dy = mesh.dy;
    D.h = S[cur][0]; D.u = S[cur][1]; D.v = S[cur][2]; D.z = z;
    D.dhdx = dbg_slp[0]; D.dudx = dbg_slp[1]; D.dvdx = dbg_slp[2]; D.dzdx = dbg_slp[3];
    D.dhdy = dbg_slp[4]; D.dudy = dbg_slp[5]; D.dvdy = dbg_slp[6]; D.dzdy = dbg_slp[7];
    D.fh = dbg_face[0]; D.fu = dbg_face[1]; D.fv = dbg_face[2]; D.fz = dbg_face[3]; D.fb = dbg_face[4];
    cudaError_t e = svk::launch_debug<T>(P, D, dbg_nh, dbg_sf, stream);
    if (e != cudaSuccess) return cuda_fail(e, "debug kernels");
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }

  // do_timestep(local_time, dt) is a function of its arguments: the scheme's own t_local and
  // dt (TemporalScheme.hpp:78) are restored afterwards.
  int do_timestep(double t_local, double dt, double* cn, int* repeat, double* new_dt) override {
    Ctl saved;
    int r = read_ctl(saved);
    if (r) return r;
    r = write_ctl_time(t_local, dt);
    if (r) return r;
    r = enqueue_timestep(false);
    if (r) return r;
    Ctl c;
    r = read_ctl(c);
    if (r) return r;
    if (cn) *cn = c.cn;
    if (repeat) *repeat = c.repeat;
    if (new_dt) *new_dt = c.new_dt;
    c.t_local = saved.t_local;
    c.dt = saved.dt;
    c.done = saved.done;
    SV_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }

  int accept() override {
    cudaError_t e = svk::launch_accept(ctl, stream);
    if (e != cudaSuccess) return cuda_fail(e, "accept kernel");
    Ctl c;
    return read_ctl(c);
  }

  int build_graph() {
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    int r0 = ensure_dev_params();
    if (r0) return r0;
    cudaGraph_t g;
    SV_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < unroll; ++i) {
      int r = enqueue_timestep(true);
      if (r) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        return r;
      }
    }
    SV_CUDA(cudaStreamEndCapture(stream, &g));
    cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    graph_dirty = false;
    return SV_OK;
  }

  // TypedTemporalScheme::step: timesteps until t_local reaches L, all on the device.
  int advance(sv_stats* out) override {
    NvtxRange nv("sv_advance");
    if (graph_dirty || !graph) {
      int r = build_graph();
      if (r) return r;
    }
    cudaError_t e = svk::launch_begin_step(ctl, 1, 0, stream);
    if (e != cudaSuccess) return cuda_fail(e, "begin step");
    SV_CUDA(cudaEventRecord(ev0, stream));
    Ctl c;
    for (long long it = 0;; ++it) {
      SV_CUDA(cudaGraphLaunch(graph, stream));
      SV_CUDA(cudaMemcpyAsync(&c, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
      SV_CUDA(cudaStreamSynchronize(stream));
      if (c.done) break;
      if (it > 100000000LL / unroll) return fail(SV_E_STATE, "step did not finish");
    }
    SV_CUDA(cudaEventRecord(ev1, stream));
    SV_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    last_advance_ms = ms;
    cur = c.cur;
    if (out) {
      out->accepted = c.step_accepted;
      out->repeated = c.step_repeated;
      out->rain_in = c.rain_in;
      out->outflow = c.outflow;
      out->wall_in = c.wall_in;
      int r = volume(&out->volume);
      if (r) return r;
    }
    if (c.error) return fail(SV_E_NONFINITE, "time became NaN: the control number was not finite");
    return SV_OK;
  }

  // Direct launches (no graph) of up to n device-controlled timesteps; with timing, every
  // kernel is bracketed by events and the per-kernel durations are summed after one sync.
  int run_timesteps(uint64_t n, int begin, sv_stats* out, int* step_done, sv_timing* timing) override {
    NvtxRange nv("sv_run_timesteps");
    if (n == 0) return fail(SV_E_ARG, "max_timesteps must be positive");
    cudaError_t e = svk::launch_begin_step(ctl, begin ? 1 : 0, (long long)n, stream);
    if (e != cudaSuccess) return cuda_fail(e, "begin step");
    std::vector<cudaEvent_t> evs;
    const int per = 2 * (N + 1);
    if (timing) {
      evs.resize(size_t(n) * per);
      for (auto& x : evs) SV_CUDA(cudaEventCreate(&x));
    }
    SV_CUDA(cudaEventRecord(ev0, stream));
    for (uint64_t i = 0; i < n; ++i) {
      int r = enqueue_timestep(true, timing ? &evs[size_t(i) * per] : nullptr);
      if (r) return r;
    }
    SV_CUDA(cudaEventRecord(ev1, stream));
    SV_CUDA(cudaEventSynchronize(ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (timing) {
      timing->total_ms = ms;
      timing->stage_ms = timing->finalize_ms = 0.0;
      timing->stage_launches = timing->finalize_launches = 0;
      for (uint64_t i = 0; i < n; ++i) {
        for (int k = 0; k <= N; ++k) {
          float d = 0.f;
          cudaEventElapsedTime(&d, evs[size_t(i) * per + 2 * k], evs[size_t(i) * per + 2 * k + 1]);
          if (k < N) { timing->stage_ms += d; timing->stage_launches++; }
          else { timing->finalize_ms += d; timing->finalize_launches++; }
        }
      }
      for (auto& x : evs) cudaEventDestroy(x);
    }
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    if (step_done) *step_done = (c.done == 1);
    if (out) {
      out->accepted = c.accepted;
      out->repeated = c.repeated;
      out->rain_in = c.rain_in;
      out->outflow = c.outflow;
      out->wall_in = c.wall_in;
      out->volume = c.volume;
    }
    if (c.error) return fail(SV_E_NONFINITE, "time became NaN: the control number was not finite");
    return SV_OK;
  }

  int set_variant(int v) override {
    if (v < 0 || v >= svk::kNumVariants) return fail(SV_E_ARG, "unknown kernel variant");
    // with tile datums only the column sweep evaluates each face in one frame (face_frame)
    if (datum && !svk::variant_is_sweep(v))
      return fail(SV_E_ARG, "tile datums need a column-sweep variant (4-10, 12-15)");
    if (svk::variant_is_fp32_only(v) && sizeof(T) != 4) return fail(SV_E_ARG, "variants 12-15 are FP32 only");
    if (svk::variant_is_split(v)) {
      int r = ensure_split();
      if (r) return r;
    }
    variant = v;
    nblk = svk::variant_partials(variant, (long long)mesh.nx, (long long)mesh.ny);
    graph_dirty = true; ++pversion;
    return SV_OK;
  }
  int get_variant() const override { return variant; }

  // Time the first-stage kernel of every variant (it reads U_[0] and writes only the stage
  // and accumulator buffers, so the state is untouched) and keep the fastest.
  int autotune(int* best_out) override {
    NvtxRange nv("sv_autotune");
    // time against a copy of the controller with `done` cleared (the live one may hold a
    // finished or paused step, which makes every stage kernel return at once)
    Ctl c;
    int r0 = read_ctl(c);
    if (r0) return r0;
    c.done = 0;
    SV_CUDA(cudaMemcpyAsync(dbg_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    svk::StageParams<T> P = base_params();
    P.ctl = dbg_ctl;
    P.stage = 0;
    P.c_s = tab.c(1);
    P.mode = svk::M_FIRST | (N == 1 ? svk::M_LAST : 0) | (diag ? svk::M_ACC : svk::M_STOREK);
    for (int j = 0; j < 4; ++j) { P.a_next[j] = 0.0; P.b[j] = 0.0; }
    if (N > 1) P.a_next[0] = tab.A(2, 1);
    for (int j = 0; j < N; ++j) P.b[j] = tab.b(j + 1);
    for (int f = 0; f < 3; ++f) {
      P.Yout[f] = Y[0][f];
      P.Kout[f] = (!diag && N > 1) ? K[0][f] : nullptr;
    }
    // the timing launches consume infiltration capacity: give them a copy
    T* cap_copy = nullptr;
    if (P.icap) {
      SV_CUDA(cudaMalloc(&cap_copy, size_t(ncells) * sizeof(T)));
      SV_CUDA(cudaMemcpyAsync(cap_copy, icap, size_t(ncells) * sizeof(T), cudaMemcpyDeviceToDevice, stream));
      P.icap = cap_copy;
    }
    struct FreeOnExit {
      T* p;
      ~FreeOnExit() { if (p) cudaFree(p); }
    } cap_guard{cap_copy};
    int best = variant;
    float best_ms = 1e30f;
    for (int v = 0; v < svk::kNumVariants; ++v) {
      if (datum && !svk::variant_is_sweep(v)) continue;
      if (svk::variant_is_fp32_only(v) && sizeof(T) != 4) continue;
      P.nblk = svk::variant_partials(v, (long long)mesh.nx, (long long)mesh.ny);
      if (!batch_path(v)) {
        int rs = ensure_strips(v);
        if (rs) return rs;
      }
      if (svk::variant_is_split(v)) {
        int rs = ensure_split();
        if (rs) return rs;
        for (int f = 0; f < 6; ++f) P.pslp[f] = pslp[f];
      }
      set_strips(P, v);
      // the batch variant runs as the batched kernel (see launch_stage_kernel): time that one
      auto launch = [&]() -> cudaError_t {
        if (!batch_path(v)) return svk::launch_variant<T>(P, v, stream);
        return svk::launch_sweep_batch<T>(d_sp + N, d_ws + 2, 1, P.nblk, pow2_mesh(), eddy_mode != SV_EDDY_OFF, stream);
      };
      if (batch_path(v)) {
        if (!d_sp) {
          SV_CUDA(alloc(&d_sp, size_t(N + 1)));
          SV_CUDA(alloc(&d_ws, size_t(4)));
        }
        long long ws[2] = {0, P.nblk};
        SV_CUDA(cudaMemcpyAsync(d_sp + N, &P, sizeof(P), cudaMemcpyHostToDevice, stream));
        SV_CUDA(cudaMemcpyAsync(d_ws + 2, ws, sizeof(ws), cudaMemcpyHostToDevice, stream));
        SV_CUDA(cudaStreamSynchronize(stream));
      }
      cudaError_t e = launch();  // warm-up
      if (e != cudaSuccess) return cuda_fail(e, "autotune launch");
      SV_CUDA(cudaEventRecord(ev0, stream));
      const int reps = 3;
      for (int i = 0; i < reps; ++i) {
        e = launch();
        if (e != cudaSuccess) return cuda_fail(e, "autotune launch");
      }
      SV_CUDA(cudaEventRecord(ev1, stream));
      SV_CUDA(cudaEventSynchronize(ev1));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev0, ev1);
      tune_ms[v] = ms / reps;
      if (ms < best_ms) { best_ms = ms; best = v; }
    }
    int r = set_variant(best);
    if (r) return r;
    if (best_out) *best_out = best;
    return SV_OK;
  }

  int volume(double* v) {
    cudaError_t e = svk::launch_volume<T>(S[cur][0], int(mesh.nx), int(mesh.ny), mesh.dx * mesh.dy, part, tile, stream);
    if (e != cudaSuccess) return cuda_fail(e, "volume kernel");
    e = svk::launch_sum(part, vol_nblk, scalar, stream);
    if (e != cudaSuccess) return cuda_fail(e, "sum kernel");
    SV_CUDA(cudaMemcpyAsync(v, scalar, sizeof(double), cudaMemcpyDeviceToHost, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }

  int set_stats(const sv_stats* in) override {
    if (!in) return fail(SV_E_ARG, "null stats");
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    c.accepted = in->accepted;
    c.repeated = in->repeated;
    c.rain_in = in->rain_in;
    c.outflow = in->outflow;
    c.wall_in = in->wall_in;
    SV_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    return SV_OK;
  }
  int get_stats(sv_stats* out) override {
    Ctl c;
    int r = read_ctl(c);
    if (r) return r;
    out->accepted = c.accepted;
    out->repeated = c.repeated;
    out->rain_in = c.rain_in;
    out->outflow = c.outflow;
    out->wall_in = c.wall_in;
    return volume(&out->volume);
  }
};


// ------------------------------------------------------------------------------------------
// Batch of independent catchments advanced together: per timestep one batched launch per RK
// stage covers every tile of every member, and one batched finalize runs every member's
// reductions and dt controller. Each member keeps its own state, dt, step clock and tallies,
// so its results are bit-identical to running it alone.
// ------------------------------------------------------------------------------------------
struct sv_batch_base {
  virtual ~sv_batch_base() {}
  std::string err;
  int fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  virtual int add(const sv_mesh_desc*, const sv_params*, int*) = 0;
  virtual int remove(int) = 0;
  virtual sv_ctx* member(int) = 0;
  virtual int advance(sv_stats*, int) = 0;
  virtual int size(int*, uint64_t*) = 0;
  virtual int set_step_limit(long long) = 0;
  virtual int status(int*, int) = 0;
  virtual int advance_steps(int, const int*, const sv_forcing*, sv_stats*, int) = 0;
  virtual int kernel_variant() const = 0;
  virtual int set_persistent(int, unsigned long long, double) = 0;
  virtual int adopt(sv_ctx*, int*) = 0;
};

template <typename T>
struct Batch final : public sv_batch_base {
  int device = 0, precision = SV_F64, rk_method = SV_RK_CLASSIC, N = 4;
  cudaStream_t stream = nullptr;
  std::vector<Solver<T>*> members;  // slot id -> member (nullptr when removed)
  // device arrays, rebuilt when membership changes
  svk::StageParams<T>* d_params = nullptr;  // [N][nact]
  svk::FinalizeParams* d_fin = nullptr;     // [nact]
  long long* d_tiles = nullptr;             // [nact + 1]
  Ctl** d_ctls = nullptr;                   // [nact]
  int* d_done = nullptr;                    // [nact]
  svk::StepQueue* d_queue = nullptr;        // [nact] steps queued by the current advance
  int nact = 0, cap = 0;
  long long total_tiles = 0;
  bool p2 = true, eddy = false, dirty = true;
  std::vector<int> active;                  // slot ids in launch order
  std::vector<unsigned long long> versions; // members' pversion at the last rebuild
  cudaGraphExec_t graph = nullptr;
  int unroll = 8;
  long long step_limit = 0;                 // timesteps per member per step (0: no limit)
  std::vector<int> last_status;             // slot id -> outcome of the last advance
  // persistent mode: one cooperative launch per advance (svk::persist_batch_kernel)
  bool persistent = false;
  unsigned long long spin_limit = 1ull << 22;  // polls without global progress before SV_E_TIMEOUT
  double max_seconds = 120.0;                  // wall-clock bound of one persistent launch
  svk::PersistMember* d_pmem = nullptr;        // [nact]
  int* d_pstatus = nullptr;                    // [0] status, then (8-byte aligned) the progress count
  unsigned long long* d_pprogress = nullptr;
  // the members' kernel variant: the column sweep of 32 rows (variant 8) in persistent mode,
  // whose strips are the persistent kernel's work items; else the batches' variant
  int member_variant() const { return persistent ? 8 : svk::batch_variant<T>(); }

  ~Batch() override {
    cudaSetDevice(device);
    if (graph) cudaGraphExecDestroy(graph);
    for (auto* m : members) delete m;
    free_arrays();
    if (stream) cudaStreamDestroy(stream);
  }
  void free_arrays() {
    cudaFree(d_params); cudaFree(d_fin); cudaFree(d_tiles); cudaFree(d_ctls); cudaFree(d_done); cudaFree(d_queue);
    cudaFree(d_pmem); cudaFree(d_pstatus); cudaFree(d_pprogress);
    d_params = nullptr; d_fin = nullptr; d_tiles = nullptr; d_ctls = nullptr; d_done = nullptr; d_queue = nullptr;
    d_pmem = nullptr; d_pstatus = nullptr; d_pprogress = nullptr;
    cap = 0;
  }
  int cuda_fail(cudaError_t e, const char* where) {
    return fail(SV_E_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  }
  int init(int prec, int rk, int dev) {
    precision = prec; rk_method = rk; device = dev;
    Tableau t;
    if (!named_tableau(rk, t)) return fail(SV_E_ARG, "unknown Runge Kutta scheme index");
    if (!is_diagonal(t)) return fail(SV_E_ARG, "batches need a tableau whose stages use only the previous stage");
    N = t.nsteps();
    SV_CUDA(cudaSetDevice(dev));
    SV_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    return SV_OK;
  }
  int add(const sv_mesh_desc* m, const sv_params* p, int* id) override {
    if (!m || !p) return fail(SV_E_ARG, "null argument");
    if (p->precision != precision || p->rk_method != rk_method)
      return fail(SV_E_ARG, "member precision and tableau must match the batch");
    auto* s = new Solver<T>();
    int r = s->init(m, p, device);
    if (r != SV_OK) {
      err = s->err;
      delete s;
      return r;
    }
    s->set_variant(member_variant());
    int slot = -1;
    for (size_t i = 0; i < members.size(); ++i)
      if (!members[i]) { slot = int(i); break; }
    if (slot < 0) { slot = int(members.size()); members.push_back(nullptr); }
    members[slot] = s;
    if (id) *id = slot;
    dirty = true;
    return SV_OK;
  }
  // a solver created and filled on its own (sv_create, then its fields) joins as a member:
  // its device memory and stream move into the batch
  int adopt(sv_ctx* c, int* id) override {
    auto* s = dynamic_cast<Solver<T>*>(c);
    if (!s || s->prm.precision != precision || s->prm.rk_method != rk_method)
      return fail(SV_E_ARG, "the solver's precision and tableau must match the batch");
    if (s->device != device) return fail(SV_E_ARG, "the solver is on another device");
    for (auto* m : members)
      if (m == s) return fail(SV_E_ARG, "the solver is already a member");
    int r = s->set_variant(member_variant());
    if (r != SV_OK) return fail(r, s->err);
    int slot = -1;
    for (size_t i = 0; i < members.size(); ++i)
      if (!members[i]) { slot = int(i); break; }
    if (slot < 0) { slot = int(members.size()); members.push_back(nullptr); }
    members[slot] = s;
    if (id) *id = slot;
    dirty = true;
    return SV_OK;
  }
  int remove(int id) override {
    if (id < 0 || id >= int(members.size()) || !members[id]) return fail(SV_E_ARG, "no such batch member");
    delete members[id];
    members[id] = nullptr;
    cudaSetDevice(device);
    dirty = true;
    return SV_OK;
  }
  sv_ctx* member(int id) override {
    if (id < 0 || id >= int(members.size()) || !members[id]) return nullptr;
    return members[id];
  }
  int size(int* n, uint64_t* bytes) override {
    int c = 0;
    uint64_t b = 0;
    for (auto* m : members)
      if (m) { ++c; b += m->device_bytes; }
    if (n) *n = c;
    if (bytes) *bytes = b;
    return SV_OK;
  }

  int rebuild() {
    active.clear();
    for (size_t i = 0; i < members.size(); ++i)
      if (members[i]) active.push_back(int(i));
    nact = int(active.size());
    if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
    if (nact > cap) {
      free_arrays();
      int c = std::max(nact, 8);
      SV_CUDA(cudaMalloc(&d_params, sizeof(svk::StageParams<T>) * size_t(N) * c));
      SV_CUDA(cudaMalloc(&d_fin, sizeof(svk::FinalizeParams) * c));
      SV_CUDA(cudaMalloc(&d_tiles, sizeof(long long) * (c + 1)));
      SV_CUDA(cudaMalloc(&d_ctls, sizeof(Ctl*) * c));
      SV_CUDA(cudaMalloc(&d_done, sizeof(int) * c));
      SV_CUDA(cudaMalloc(&d_queue, sizeof(svk::StepQueue) * c));
      SV_CUDA(cudaMalloc(&d_pmem, sizeof(svk::PersistMember) * c));
      SV_CUDA(cudaMalloc(&d_pstatus, sizeof(int)));
      SV_CUDA(cudaMalloc(&d_pprogress, sizeof(unsigned long long)));
      cap = c;
    }
    std::vector<svk::StageParams<T>> hp(size_t(N) * std::max(nact, 1));
    std::vector<svk::FinalizeParams> hf(std::max(nact, 1));
    std::vector<long long> ht(nact + 1, 0);
    std::vector<Ctl*> hc(std::max(nact, 1));
    p2 = true;
    eddy = false;
    for (int k = 0; k < nact; ++k) {
      Solver<T>* m = members[active[k]];
      // the tile prefix and the partials follow the batch kernel's decomposition
      if (m->variant != member_variant()) m->set_variant(member_variant());
      if (persistent) {  // the persistent kernel runs each member's interior strips in the interior sweep
        int rs = m->ensure_strips(member_variant());
        if (rs) return fail(rs, "member " + std::to_string(active[k]) + ": " + m->err);
      }
      ht[k + 1] = ht[k] + m->nblk;
      int e2;
      p2 = p2 && std::frexp(m->mesh.dx, &e2) == 0.5 && std::frexp(m->mesh.dy, &e2) == 0.5;
      eddy = eddy || m->eddy_mode != SV_EDDY_OFF;
      for (int st = 0; st < N; ++st) hp[size_t(st) * nact + k] = m->stage_params(st);
      hf[k] = m->finalize_params(true);
      hf[k].q = d_queue + k;
      hf[k].fc = m->fc;
      hc[k] = m->ctl;
    }
    total_tiles = ht[nact];
    versions.assign(nact, 0);
    for (int k = 0; k < nact; ++k) versions[k] = members[active[k]]->pversion;
    if (nact > 0) {
      SV_CUDA(cudaMemcpyAsync(d_params, hp.data(), sizeof(svk::StageParams<T>) * size_t(N) * nact,
                              cudaMemcpyHostToDevice, stream));
      SV_CUDA(cudaMemcpyAsync(d_fin, hf.data(), sizeof(svk::FinalizeParams) * nact, cudaMemcpyHostToDevice, stream));
      SV_CUDA(cudaMemcpyAsync(d_tiles, ht.data(), sizeof(long long) * (nact + 1), cudaMemcpyHostToDevice, stream));
      SV_CUDA(cudaMemcpyAsync(d_ctls, hc.data(), sizeof(Ctl*) * nact, cudaMemcpyHostToDevice, stream));
      SV_CUDA(cudaStreamSynchronize(stream));
    }
    dirty = false;
    return SV_OK;
  }

  int enqueue_timestep() {
    for (int st = 0; st < N; ++st) {
      cudaError_t e = svk::variant_is_sweep(svk::batch_variant<T>())
                          ? svk::launch_sweep_batch<T>(d_params + size_t(st) * nact, d_tiles, nact, total_tiles, p2,
                                                       eddy, stream)
                          : svk::launch_stage_batch<T>(d_params + size_t(st) * nact, d_tiles, nact, total_tiles, p2,
                                                       eddy, stream);
      if (e != cudaSuccess) return cuda_fail(e, "batched stage kernel");
    }
    cudaError_t e = svk::launch_finalize_batch(d_fin, nact, stream);
    if (e != cudaSuccess) return cuda_fail(e, "batched finalize kernel");
    return SV_OK;
  }

  int build_graph() {
    cudaGraph_t g;
    SV_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < unroll; ++i) {
      int r = enqueue_timestep();
      if (r) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        return r;
      }
    }
    SV_CUDA(cudaStreamEndCapture(stream, &g));
    cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
    return SV_OK;
  }

  // Brings the launch arrays and the graph up to date with the membership.
  int prepare() {
    SV_CUDA(cudaSetDevice(device));
    for (size_t k = 0; k < active.size() && !dirty; ++k)
      if (!members[active[k]] || members[active[k]]->pversion != versions[k]) dirty = true;
    if (dirty) {
      int r = rebuild();
      if (r) return r;
    }
    if (nact == 0) return SV_OK;
    // members' own streams may hold pending uploads (set_field/set_forcing synchronise, but
    // be safe): order them before the batch's work
    for (int k : active) SV_CUDA(cudaStreamSynchronize(members[k]->stream));
    if (!graph && !persistent) {
      int r = build_graph();
      if (r) return r;
    }
    return SV_OK;
  }

  // Runs the queued steps of every member (hq[k] for active member k) to completion: one
  // upload of the queues, graph launches of `unroll` timesteps until every member is done,
  // one read-back. Each member runs its steps back to back at its own pace; a failing
  // member stops alone. hq receives the per-step results; last_status each slot's outcome.
  int run_queue(std::vector<svk::StepQueue>& hq) {
    NvtxRange nv(persistent ? "sv_batch_advance (persistent)" : "sv_batch_advance");
    SV_CUDA(cudaMemcpyAsync(d_queue, hq.data(), sizeof(svk::StepQueue) * nact, cudaMemcpyHostToDevice, stream));
    cudaError_t e = svk::launch_begin_queue(d_fin, nact, stream);
    if (e != cudaSuccess) return cuda_fail(e, "begin queued steps");
    std::vector<int> done(nact);
    if (persistent) {
      // every member's queued steps in one cooperative launch
      e = svk::launch_persist_init(d_fin, d_pmem, d_tiles, nact, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(d_pstatus, 0, sizeof(int), stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(d_pprogress, 0, sizeof(unsigned long long), stream);
      svk::PersistParams<T> PP{};
      PP.Ps = d_params;
      PP.Fs = d_fin;
      PP.mem = d_pmem;
      PP.nact = nact;
      PP.nstages = N;
      PP.status = d_pstatus;
      PP.progress = d_pprogress;
      PP.spin_limit = spin_limit;
      PP.max_ns = (unsigned long long)(max_seconds * 1e9);
      if (e == cudaSuccess) e = svk::launch_persist<T>(PP, p2, eddy, stream);
      if (e != cudaSuccess) return cuda_fail(e, "persistent batch kernel");
      int st = 0;
      SV_CUDA(cudaMemcpyAsync(&st, d_pstatus, sizeof(int), cudaMemcpyDeviceToHost, stream));
      SV_CUDA(cudaStreamSynchronize(stream));
      if (st != 0) {
        // the members keep the state of their last completed timestep (a timestep's result
        // replaces U_[0] only in its finalize)
        for (int k = 0; k < nact; ++k) {  // the host mirrors of the state parity
          Ctl c;
          int r = members[active[k]]->read_ctl(c);
          if (r) return fail(r, members[active[k]]->err);
        }
        last_status.assign(members.size(), SV_E_TIMEOUT);
        return fail(SV_E_TIMEOUT, "persistent batch kernel gave up: no work item completed during " +
                                      std::to_string(spin_limit) + " polls, or the launch ran past " +
                                      std::to_string(max_seconds) + " s");
      }
    }
    for (long long it = 0; !persistent; ++it) {
      SV_CUDA(cudaGraphLaunch(graph, stream));
      e = svk::launch_gather_done(d_ctls, nact, d_done, stream);
      if (e != cudaSuccess) return cuda_fail(e, "gather done");
      SV_CUDA(cudaMemcpyAsync(done.data(), d_done, sizeof(int) * nact, cudaMemcpyDeviceToHost, stream));
      SV_CUDA(cudaStreamSynchronize(stream));
      bool all = true;
      for (int d : done) all = all && d != 0;
      if (all) break;
      if (it > 100000000LL / unroll) return fail(SV_E_STATE, "batch step did not finish");
    }
    SV_CUDA(cudaMemcpyAsync(hq.data(), d_queue, sizeof(svk::StepQueue) * nact, cudaMemcpyDeviceToHost, stream));
    SV_CUDA(cudaStreamSynchronize(stream));
    int n_nan = 0, n_limit = 0;
    last_status.assign(members.size(), SV_OK);
    for (int k = 0; k < nact; ++k) {
      members[active[k]]->cur = hq[k].cur;  // the state parity moved on the device
      last_status[active[k]] = hq[k].status;
      n_nan += hq[k].status == SV_E_NONFINITE;
      n_limit += hq[k].status == SV_E_LIMIT;
    }
    if (n_nan)
      return fail(SV_E_NONFINITE, std::to_string(n_nan) + " member(s)' time became NaN: the control number was not "
                                  "finite (sv_batch_status names them; the other members completed their steps)");
    if (n_limit)
      return fail(SV_E_LIMIT, std::to_string(n_limit) + " member(s) reached the step limit of " +
                                  std::to_string(step_limit) + " timesteps before the end of a step "
                                  "(sv_batch_status names them; the other members completed their steps)");
    return SV_OK;
  }

  static void step_stats(const svk::StepQueue& q, int s, sv_stats& o) {
    o.accepted = q.acc[s];
    o.repeated = q.rep[s];
    o.rain_in = q.rain[s];
    o.outflow = q.outflow[s];
    o.wall_in = q.wall[s];
    o.volume = q.volume[s];
  }

  // One step (of each member's own length L) for every member, with the forcing each member
  // holds, in batched launches.
  int advance(sv_stats* out, int n_out) override {
    int r = prepare();
    if (r || nact == 0) return r;
    std::vector<svk::StepQueue> hq(nact);
    for (auto& q : hq) {
      q = svk::StepQueue{};
      q.n = 1;
      q.keep_first = 1;
      q.limit = step_limit;
    }
    int rc = run_queue(hq);
    if (rc == SV_E_CUDA || rc == SV_E_STATE) return rc;
    for (int k = 0; k < nact; ++k)
      if (out && active[k] < n_out) step_stats(hq[k], 0, out[active[k]]);
    return rc;
  }

  // Up to kMaxQueuedSteps steps per member in one call (TypedTemporalScheme::solve over
  // several steps): member id runs nsteps[id] steps with forcing[id * max_steps + s].
  int advance_steps(int max_steps, const int* nsteps, const sv_forcing* forcing, sv_stats* out, int n) override {
    if (max_steps < 1 || max_steps > svk::kMaxQueuedSteps)
      return fail(SV_E_LIMIT, "at most " + std::to_string(svk::kMaxQueuedSteps) + " steps per batched advance");
    if (n < 0 || (n > 0 && (!nsteps || !forcing))) return fail(SV_E_ARG, "null step counts or forcing");
    int r = prepare();
    if (r || nact == 0) return r;
    std::vector<svk::StepQueue> hq(nact);
    for (int k = 0; k < nact; ++k) {
      svk::StepQueue& q = hq[k];
      q = svk::StepQueue{};
      q.limit = step_limit;
      const int id = active[k];
      const int ns = id < n ? nsteps[id] : 0;
      if (ns < 0 || ns > max_steps) return fail(SV_E_ARG, "step count of member " + std::to_string(id) + " out of range");
      q.n = ns;
      for (int st = 0; st < ns; ++st) {
        int e = members[id]->make_forcing(&forcing[size_t(id) * max_steps + st], &q.f[st], false);
        if (e) return fail(e, "member " + std::to_string(id) + ", step " + std::to_string(st) + ": " + members[id]->err);
      }
    }
    int rc = run_queue(hq);
    if (rc == SV_E_CUDA || rc == SV_E_STATE) return rc;
    if (out)
      for (int k = 0; k < nact; ++k) {
        const int id = active[k];
        if (id >= n) continue;
        for (int st = 0; st < max_steps; ++st) {
          sv_stats& o = out[size_t(id) * max_steps + st];
          o = sv_stats{};
          if (st < hq[k].n && st <= hq[k].k && (st < hq[k].k || hq[k].status != 0)) step_stats(hq[k], st, o);
        }
      }
    return rc;
  }

  int kernel_variant() const override { return member_variant(); }

  int set_persistent(int on, unsigned long long limit, double seconds) override {
    persistent = on != 0;
    spin_limit = limit ? limit : (1ull << 22);
    max_seconds = seconds > 0.0 ? seconds : 120.0;
    dirty = true;
    return SV_OK;
  }

  int set_step_limit(long long n) override {
    if (n < 0) return fail(SV_E_ARG, "step limit must be >= 0");
    step_limit = n;
    return SV_OK;
  }
  int status(int* out, int n) override {
    if (!out || n < 0) return fail(SV_E_ARG, "null status array");
    for (int i = 0; i < n; ++i) out[i] = i < int(last_status.size()) ? last_status[i] : SV_OK;
    return SV_OK;
  }
};

}  // namespace

struct sv_batch {
  std::unique_ptr<sv_batch_base> impl;
};

extern "C" {

int sv_create(const sv_mesh_desc* mesh, const sv_params* params, int device, sv_ctx** out) {
  if (!mesh || !params || !out) {
    g_create_err = "null argument";
    return SV_E_ARG;
  }
  *out = nullptr;
  sv_ctx* c = nullptr;
  int r;
  if (params->precision == SV_F64) {
    auto* s = new Solver<double>();
    r = s->init(mesh, params, device);
    c = s;
  } else if (params->precision == SV_F32 || params->precision == SV_F32_DATUM64) {
    auto* s = new Solver<float>();
    r = s->init(mesh, params, device);
    c = s;
  } else {
    g_create_err = "precision not available";
    return SV_E_ARG;
  }
  if (r != SV_OK) {
    g_create_err = c->err;
    delete c;
    return r;
  }
  *out = c;
  return SV_OK;
}

void sv_destroy(sv_ctx* ctx) { delete ctx; }

#define SV_CHECK_CTX(ctx) \
  if (!(ctx)) return SV_E_ARG

int sv_set_field(sv_ctx* ctx, int id, const double* host, uint64_t n) { SV_CHECK_CTX(ctx); return ctx->set_field(id, host, n); }
int sv_get_field(sv_ctx* ctx, int id, double* host, uint64_t n) { SV_CHECK_CTX(ctx); return ctx->get_field(id, host, n); }
int sv_set_manning(sv_ctx* ctx, double a, double b, double c, double d) { SV_CHECK_CTX(ctx); return ctx->set_manning(a, b, c, d); }
int sv_set_eddy_viscosity(sv_ctx* ctx, int mode, double mu, double mu_const, double mu_smag) {
  SV_CHECK_CTX(ctx);
  return ctx->set_eddy(mode, mu, mu_const, mu_smag);
}
int sv_set_source_order(sv_ctx* ctx, const int* terms, int n) { SV_CHECK_CTX(ctx); return ctx->set_source_order(terms, n); }
int sv_set_forcing(sv_ctx* ctx, const sv_forcing* f) { SV_CHECK_CTX(ctx); return ctx->set_forcing(f); }
int sv_set_dt(sv_ctx* ctx, double dt) { SV_CHECK_CTX(ctx); return ctx->set_dt(dt); }
int sv_get_dt(sv_ctx* ctx, double* dt) { SV_CHECK_CTX(ctx); if (!dt) return SV_E_ARG; return ctx->get_dt(dt); }
int sv_eval_dudt(sv_ctx* ctx, int s, double t, double dt) { SV_CHECK_CTX(ctx); return ctx->eval_dudt(s, t, dt); }
int sv_do_timestep(sv_ctx* ctx, double t, double dt, double* cn, int* rep, double* nd) {
  SV_CHECK_CTX(ctx);
  return ctx->do_timestep(t, dt, cn, rep, nd);
}
int sv_accept(sv_ctx* ctx) { SV_CHECK_CTX(ctx); return ctx->accept(); }
int sv_advance(sv_ctx* ctx, sv_stats* out) { SV_CHECK_CTX(ctx); return ctx->advance(out); }
int sv_get_stats(sv_ctx* ctx, sv_stats* out) { SV_CHECK_CTX(ctx); if (!out) return SV_E_ARG; return ctx->get_stats(out); }
int sv_set_stats(sv_ctx* ctx, const sv_stats* in) { SV_CHECK_CTX(ctx); return ctx->set_stats(in); }
int sv_run_timesteps(sv_ctx* ctx, uint64_t n, int begin, sv_stats* out, int* step_done, sv_timing* t) {
  SV_CHECK_CTX(ctx);
  return ctx->run_timesteps(n, begin, out, step_done, t);
}
int sv_batch_create(int precision, int rk_method, int device, sv_batch** out) {
  if (!out) return SV_E_ARG;
  *out = nullptr;
  std::unique_ptr<sv_batch_base> b;
  int r;
  if (precision == SV_F64) {
    auto* x = new Batch<double>();
    b.reset(x);
    r = x->init(precision, rk_method, device);
  } else if (precision == SV_F32 || precision == SV_F32_DATUM64) {
    auto* x = new Batch<float>();
    b.reset(x);
    r = x->init(precision, rk_method, device);
  } else {
    g_create_err = "precision not available";
    return SV_E_ARG;
  }
  if (r != SV_OK) {
    g_create_err = b->err;
    return r;
  }
  *out = new sv_batch{std::move(b)};
  return SV_OK;
}
void sv_batch_destroy(sv_batch* b) { delete b; }
int sv_batch_add(sv_batch* b, const sv_mesh_desc* m, const sv_params* p, int* id) {
  if (!b) return SV_E_ARG;
  int r = b->impl->add(m, p, id);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_adopt(sv_batch* b, sv_ctx* solver, int* id) {
  if (!b || !solver) return SV_E_ARG;
  int r = b->impl->adopt(solver, id);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_remove(sv_batch* b, int id) {
  if (!b) return SV_E_ARG;
  int r = b->impl->remove(id);
  if (r) g_create_err = b->impl->err;
  return r;
}
sv_ctx* sv_batch_member(sv_batch* b, int id) { return b ? b->impl->member(id) : nullptr; }
int sv_batch_advance(sv_batch* b, sv_stats* out, int n_out) {
  if (!b) return SV_E_ARG;
  int r = b->impl->advance(out, n_out);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_set_step_limit(sv_batch* b, long long max_timesteps) {
  if (!b) return SV_E_ARG;
  int r = b->impl->set_step_limit(max_timesteps);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_advance_steps(sv_batch* b, int max_steps, const int* nsteps, const sv_forcing* forcing, sv_stats* out,
                           int n) {
  if (!b) return SV_E_ARG;
  int r = b->impl->advance_steps(max_steps, nsteps, forcing, out, n);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_set_persistent(sv_batch* b, int on, uint64_t spin_limit, double max_seconds) {
  if (!b) return SV_E_ARG;
  return b->impl->set_persistent(on, spin_limit, max_seconds);
}
int sv_batch_kernel_variant(sv_batch* b, int* variant) {
  if (!b || !variant) return SV_E_ARG;
  *variant = b->impl->kernel_variant();
  return SV_OK;
}
int sv_batch_status(sv_batch* b, int* status, int n) {
  if (!b) return SV_E_ARG;
  int r = b->impl->status(status, n);
  if (r) g_create_err = b->impl->err;
  return r;
}
int sv_batch_size(sv_batch* b, int* n, uint64_t* bytes) {
  if (!b) return SV_E_ARG;
  return b->impl->size(n, bytes);
}

int sv_set_kernel_variant(sv_ctx* ctx, int v) { SV_CHECK_CTX(ctx); return ctx->set_variant(v); }
int sv_get_kernel_variant(sv_ctx* ctx, int* v) { SV_CHECK_CTX(ctx); if (!v) return SV_E_ARG; *v = ctx->get_variant(); return SV_OK; }
int sv_autotune(sv_ctx* ctx, int* best) { SV_CHECK_CTX(ctx); return ctx->autotune(best); }
int sv_get_autotune_ms(sv_ctx* ctx, float* ms, int n) {
  SV_CHECK_CTX(ctx);
  if (!ms || n < 0) return SV_E_ARG;
  for (int v = 0; v < n; ++v) ms[v] = ctx->autotune_ms(v);
  return SV_OK;
}
int sv_last_advance_ms(sv_ctx* ctx, double* ms) { SV_CHECK_CTX(ctx); if (!ms) return SV_E_ARG; *ms = ctx->last_advance_ms; return SV_OK; }
const char* sv_last_error(const sv_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_err.c_str(); }

}  // extern "C"
