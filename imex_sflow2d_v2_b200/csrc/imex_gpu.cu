// imex_gpu.cu -- C ABI of the sm_100a IMEX_SfloW2D time step (include/imex_gpu.h).
//
// One context = one CUDA stream + device-resident state (SoA planes), static
// planes, and a device clock.  The per-routine entry points mirror the
// reference driver's calls (check_solve, timestep, imex_RK_solver,
// update_erosion_deposition_cell); imex_gpu_advance runs the whole driver loop
// body on the device and can replay it from a captured CUDA graph.
#include <cuda_runtime.h>

// namespace of this unit's copy of the kernels (imex_device.cuh)
#define IMEX_TU_NS tu_gpu

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/imex_gpu.h"
#include "imex_kernels.cuh"
#include "imex_batch_api.h"
#include "imex_mlp.cuh"
#include "imex_setup.cuh"
#include "imex_output.cuh"
#include "imex_fortran_fmt.h"

using namespace imex;

struct ImexCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;  // created by the context
  // host-state steps (imex_gpu_advance_host): the transfer stream and its
  // band events, created on first use
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> band_ev;
  // tensor map of q for the flux kernel's TMA tile loads (k_flux_tma)
  alignas(64) CUtensorMap q_tmap{};
  bool q_tmap_ok = false;
  DevParams P{};
  DevParams* dP = nullptr;      // device copy of P
  ImexParams host_params{};
  int ns = 1;
  // device buffers
  double* q = nullptr;     // nv planes
  double* X = nullptr;     // nv planes: stage-1 divFlux - expl_terms
  uint8_t* mask = nullptr;
  uint8_t* cellinfo = nullptr;
  double *Bx = nullptr, *By = nullptr, *Bxx = nullptr, *Bxy = nullptr, *Byy = nullptr;
  double *gc = nullptr, *dgc = nullptr, *gcsx = nullptr, *gcsy = nullptr;
  double* release = nullptr;
  double *erodible = nullptr, *deposit = nullptr, *erosion = nullptr, *Bcent = nullptr;
  RingCell* ring = nullptr;
  DevClock* clk = nullptr;
  DevClock* clk_host = nullptr;  // pinned mirror
  double* scratch = nullptr;     // AoS staging for transfers
  NewtonWork nw{};               // stage-2 Newton state between passes
  // driver output sweep (imex_gpu_post_init): planes, levels, diag partials
  bool post_on = false;
  PostLevels post_levels{};
  PostPlanes post{};
  double* post_buf = nullptr;
  uint32_t* post_vuln = nullptr;
  double* post_diag = nullptr;
  double* nw_buf = nullptr;      // backing store of nw's FP64 planes
  uint32_t* nw_lists = nullptr;  // backing store of nw's three cell lists
  // learned warm start and training-pair harvest
  struct ImexMLP* warm_mlp = nullptr;  // not owned
  uint32_t* nw_wlist = nullptr;
  float* nw_feat = nullptr;
  double* nw_guess = nullptr;
  float* h_x = nullptr;
  float* h_y = nullptr;
  // output_solution writer (imex_gpu_output): device planes, pinned staging,
  // the event after the staging copies and the host thread that formats
  std::thread out_thread;
  bool out_pending = false;
  int out_status = 0;
  std::string out_error;
  double* out_dev = nullptr;
  size_t out_dev_n = 0;
  double* out_host = nullptr;
  size_t out_host_n = 0;
  cudaEvent_t out_ev = nullptr;
  size_t scratch_bytes = 0;
  bool x_valid = false;          // X holds the fluxes of the current state
  bool exchange = false;         // erosion/deposition planes present
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int64_t graph_launches = 0;    // kernels in one replay of graph_exec
  int64_t launches = 0;
  uint32_t error_mask_acc = 0;
  std::string last_error;
  // per-kernel CUDA-event timing (imex_gpu_profile)
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;  // kernel id, events
  size_t ev_used = 0;
};

namespace {

int fail(ImexCtx* c, int code, const std::string& msg) {
  if (c) c->last_error = msg;
  return code;
}

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      return fail(ctx, IMEX_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    }                                                                         \
  } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t n) {
  return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
}

int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }

// Function attributes belong to a device: `mask` records, per device
// index, that the attribute has been set there.  Host threads may race to
// set the same attribute; setting it twice is harmless, and the mask is an
// atomic so that the record itself is well defined.
bool attr_needed(std::atomic<unsigned long long>& mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
  return (mask.load(std::memory_order_acquire) & (1ULL << dev)) == 0;
}
void attr_done(std::atomic<unsigned long long>& mask) {
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64)
    mask.fetch_or(1ULL << dev, std::memory_order_acq_rel);
}

// Upload an (nx,ny) Fortran plane into a pitched device plane.
cudaError_t upload_plane(ImexCtx* ctx, double* dst, const double* src, double fill) {
  const int nx = ctx->P.nx, ny = ctx->P.ny;
  const int64_t pitch = ctx->P.pitch;
  std::vector<double> h((size_t)ctx->P.plane, fill);
  if (src)
    for (int k = 0; k < ny; ++k) std::memcpy(&h[(size_t)k * pitch], src + (size_t)k * nx, nx * sizeof(double));
  return cudaMemcpy(dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
}

dim3 tile_grid(const DevParams& P) { return dim3((P.nx + TX - 1) / TX, (P.ny + TY - 1) / TY); }

int grid_1d(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 64);
}

// Kernel ids for imex_gpu_kernel_times.
enum {
  KID_MASK = 0,
  KID_FLUX = 1,
  KID_S2_FIRST = 2,   // stage 2 up to Newton iteration 1
  KID_S2_ITER = 3,    // Newton iterations 2.. (both list passes and the tail)
  KID_S2_POST = 4,    // sign guard and assembly
  KID_EROSION = 5,
  KID_N = 6
};

cudaEvent_t pool_event(ImexCtx* ctx) {
  if (ctx->ev_used == ctx->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    ctx->ev_pool.push_back(e);
  }
  return ctx->ev_pool[ctx->ev_used++];
}

struct ProfScope {
  ImexCtx* ctx;
  int kid;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(ImexCtx* c, int k) : ctx(c), kid(k) {
    if (ctx->prof) {
      a = pool_event(ctx);
      b = pool_event(ctx);
      cudaEventRecord(a, ctx->stream);
    }
  }
  ~ProfScope() {
    if (ctx->prof) {
      cudaEventRecord(b, ctx->stream);
      ctx->ev_pending.push_back({kid, {a, b}});
    }
  }
};

// ------------------------------------------------------- launch helpers
// The tensor map of q for k_flux_tma: dims {nx, ny, n_v} in elements, row
// and plane strides in bytes (multiples of 16: the pitch is a multiple of
// 16 elements), box {SW, SH, n_v} = the flux tile with its halo, zero fill
// outside the grid.  The encoder comes from the driver through the
// runtime; without it (or if it refuses the map) k_flux loads the tile
// itself.
bool encode_q_map(ImexCtx* ctx) {
  typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                    const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                    const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult qr;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) !=
          cudaSuccess ||
      qr != cudaDriverEntryPointSuccess || !fn)
    return false;
  const DevParams& P = ctx->P;
  if ((P.pitch * sizeof(double)) % 16 != 0 || (reinterpret_cast<uintptr_t>(ctx->q) % 16) != 0)
    return false;
  const cuuint64_t dims[3] = {(cuuint64_t)P.nx, (cuuint64_t)P.ny, (cuuint64_t)P.nv};
  const cuuint64_t strides[2] = {(cuuint64_t)P.pitch * sizeof(double),
                                 (cuuint64_t)P.plane * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)SW, (cuuint32_t)SH, (cuuint32_t)P.nv};
  const cuuint32_t elem[3] = {1, 1, 1};
  const CUresult r = reinterpret_cast<EncodeTiledFn>(fn)(
      &ctx->q_tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ctx->q, dims, strides, box, elem,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int NS>
cudaError_t launch_flux_ns(ImexCtx* ctx) {
  const DevParams& P = ctx->P;
  size_t smem = sizeof(FluxShared<NS>);
  if (ctx->q_tmap_ok) {
    static std::atomic<unsigned long long> attr_tma{0};
    if (attr_needed(attr_tma)) {
      cudaError_t e = cudaFuncSetAttribute(k_flux_tma<NS>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(k_flux_tma<NS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                               (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return e;
      attr_done(attr_tma);
    }
    k_flux_tma<NS><<<tile_grid(P), FLUX_THREADS, smem, ctx->stream>>>(
        ctx->P, ctx->q_tmap, ctx->q, ctx->mask, ctx->cellinfo, ctx->Bx, ctx->By, ctx->Bxx,
        ctx->Bxy, ctx->Byy, ctx->gc, ctx->dgc, ctx->gcsx, ctx->gcsy, ctx->ring, ctx->clk, ctx->X);
    ctx->launches += 1;
    return cudaGetLastError();
  }
  static std::atomic<unsigned long long> attr_set{0};
  if (attr_needed(attr_set)) {
    cudaError_t e = cudaFuncSetAttribute(k_flux<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_flux<NS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    attr_done(attr_set);
  }
  k_flux<NS><<<tile_grid(P), FLUX_THREADS, smem, ctx->stream>>>(
      ctx->P, ctx->q, ctx->mask, ctx->cellinfo, ctx->Bx, ctx->By, ctx->Bxx, ctx->Bxy, ctx->Byy,
      ctx->gc, ctx->dgc, ctx->gcsx, ctx->gcsy, ctx->ring, ctx->clk, ctx->X);
  ctx->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_flux(ImexCtx* ctx) {
  switch (ctx->ns) {
    case 1: return launch_flux_ns<1>(ctx);
    case 2: return launch_flux_ns<2>(ctx);
    case 3: return launch_flux_ns<3>(ctx);
    default: return launch_flux_ns<4>(ctx);
  }
}

cudaError_t launch_warm_predict(ImexCtx* ctx);  // after ImexMLP (below)

template <int NS>
cudaError_t launch_stage2_ns(ImexCtx* ctx) {
  const DevParams& P = ctx->P;
  const long long ncell = (long long)P.nx * P.ny;
  const int grid = grid_1d(ncell, STAGE2_THREADS);
  // list passes: one resident wave (IMEX_STAGE2_MINB blocks per SM), grid-stride
  const int lgrid = std::min(grid, 148 * IMEX_STAGE2_MINB);
  k_nw_reset<<<1, 1, 0, ctx->stream>>>(ctx->clk);
  {
    ProfScope ps(ctx, KID_S2_FIRST);
    k_stage2_first<NS><<<grid, STAGE2_THREADS, 0, ctx->stream>>>(
        ctx->P, ctx->q, ctx->X, ctx->mask, ctx->Bx, ctx->By, ctx->Bxx, ctx->Bxy, ctx->Byy,
        ctx->gc, ctx->nw, ctx->clk);
    if (ctx->nw.warm) {
      cudaError_t e = launch_warm_predict(ctx);
      if (e != cudaSuccess) return e;
      k_stage2_wstart<NS><<<lgrid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx,
                                                                     ctx->By, ctx->nw, ctx->clk);
      ctx->launches += 1;
    }
  }
  {
    ProfScope ps(ctx, KID_S2_ITER);
    k_stage2_iter<NS><<<lgrid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx,
                                                                 ctx->By, ctx->nw, ctx->clk, 2);
    k_stage2_iter<NS><<<lgrid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx,
                                                                 ctx->By, ctx->nw, ctx->clk, 3);
    k_stage2_tail<NS><<<lgrid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx,
                                                                 ctx->By, ctx->nw, ctx->clk);
    if (ctx->nw.warm) {
      k_stage2_fallback<NS><<<lgrid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx,
                                                                       ctx->By, ctx->nw, ctx->clk);
      ctx->launches += 1;
    }
  }
  if (ctx->nw.harvest) {
    k_harvest<NS><<<grid_1d(ncell, 128), 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->Bx, ctx->By,
                                                                ctx->nw, ctx->clk);
    ctx->launches += 1;
  }
  {
    ProfScope ps(ctx, KID_S2_POST);
    k_stage2_post<NS><<<grid, STAGE2_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask,
                                                                ctx->cellinfo, ctx->nw, ctx->clk);
  }
  ctx->launches += 6;
  return cudaGetLastError();
}

cudaError_t launch_stage2(ImexCtx* ctx) {
  switch (ctx->ns) {
    case 1: return launch_stage2_ns<1>(ctx);
    case 2: return launch_stage2_ns<2>(ctx);
    case 3: return launch_stage2_ns<3>(ctx);
    default: return launch_stage2_ns<4>(ctx);
  }
}

template <int NS>
cudaError_t launch_erosion_ns(ImexCtx* ctx) {
  const DevParams& P = ctx->P;
  int grid = grid_1d((long long)P.nx * P.ny, 128);
  k_erosion<NS><<<grid, 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask, ctx->Bx, ctx->By,
                                               ctx->erodible, ctx->deposit, ctx->erosion,
                                               ctx->Bcent, ctx->clk);
  ctx->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_erosion(ImexCtx* ctx) {
  switch (ctx->ns) {
    case 1: return launch_erosion_ns<1>(ctx);
    case 2: return launch_erosion_ns<2>(ctx);
    case 3: return launch_erosion_ns<3>(ctx);
    default: return launch_erosion_ns<4>(ctx);
  }
}

// topography_reconstruction on the device after a bed change
cudaError_t launch_topo(ImexCtx* ctx) {
  const DevParams& P = ctx->P;
  const long long n = (long long)P.nx * P.ny;
  k_topo_geom<<<grid_1d(n, 256), 256, 0, ctx->stream>>>(ctx->P, ctx->Bcent, ctx->Bx, ctx->By,
                                                         ctx->Bxx, ctx->Bxy, ctx->Byy);
  ctx->launches += 1;
  if (P.slope_correction_flag) {
    const long long m = n + (long long)(P.nx + 1) * P.ny + (long long)P.nx * (P.ny + 1);
    k_topo_gc<<<grid_1d(m, 256), 256, 0, ctx->stream>>>(ctx->P, ctx->Bx, ctx->By, ctx->Bxx,
                                                         ctx->Bxy, ctx->gc, ctx->dgc, ctx->gcsx,
                                                         ctx->gcsy);
    ctx->launches += 1;
  }
  return cudaGetLastError();
}

cudaError_t launch_post_sweep(ImexCtx* ctx, int init) {
  const DevParams& P = ctx->P;
  const int grid = grid_1d((long long)P.nx * P.ny, 128);
  switch (ctx->ns) {
    case 1: k_post_sweep<1><<<grid, 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask, ctx->post, ctx->post_levels, init); break;
    case 2: k_post_sweep<2><<<grid, 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask, ctx->post, ctx->post_levels, init); break;
    case 3: k_post_sweep<3><<<grid, 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask, ctx->post, ctx->post_levels, init); break;
    default: k_post_sweep<4><<<grid, 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->mask, ctx->post, ctx->post_levels, init); break;
  }
  ctx->launches += 1;
  return cudaGetLastError();
}

constexpr int DIAG_BLOCKS = 148 * 4;

cudaError_t launch_post_diag(ImexCtx* ctx) {
  double* part = ctx->post_diag + 4;
  switch (ctx->ns) {
    case 1: k_post_diag<1><<<DIAG_BLOCKS, DIAG_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->post.qp_h, part); break;
    case 2: k_post_diag<2><<<DIAG_BLOCKS, DIAG_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->post.qp_h, part); break;
    case 3: k_post_diag<3><<<DIAG_BLOCKS, DIAG_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->post.qp_h, part); break;
    default: k_post_diag<4><<<DIAG_BLOCKS, DIAG_THREADS, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->post.qp_h, part); break;
  }
  k_post_diag_fold<<<1, 32, 0, ctx->stream>>>(part, DIAG_BLOCKS, ctx->post_diag);
  ctx->launches += 2;
  return cudaGetLastError();
}

cudaError_t launch_mask(ImexCtx* ctx, int solve_all = 0) {
  const DevParams& P = ctx->P;
  k_mask<<<tile_grid(P), 256, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->release, ctx->cellinfo,
                                                ctx->clk, ctx->mask, ctx->clk, solve_all);
  ctx->launches += 1;
  return cudaGetLastError();
}

bool erosion_active(const ImexCtx* ctx) {
  const ImexParams& p = ctx->host_params;
  return p.erosion_coeff != 0.0 || p.settling_flag || p.entrainment_flag;
}

// Device part of one driver-loop pass: mask, fluxes + CFL, dt clip, stage 2
// , erosion/deposition, t += dt.
cudaError_t enqueue_step(ImexCtx* ctx) {
  cudaError_t e;
  k_step_begin<<<1, 1, 0, ctx->stream>>>(ctx->clk, ctx->P.max_dt, 1);
  ctx->launches += 1;
  {
    ProfScope ps(ctx, KID_MASK);
    if ((e = launch_mask(ctx)) != cudaSuccess) return e;
  }
  {
    ProfScope ps(ctx, KID_FLUX);
    if ((e = launch_flux(ctx)) != cudaSuccess) return e;
  }
  k_dt_clip<<<1, 1, 0, ctx->stream>>>(ctx->clk, 1);
  ctx->launches += 1;
  if ((e = launch_stage2(ctx)) != cudaSuccess) return e;
  if (erosion_active(ctx)) {
    ProfScope ps(ctx, KID_EROSION);
    if ((e = launch_erosion(ctx)) != cudaSuccess) return e;
  }
  if (ctx->P.topo_change_flag && (e = launch_topo(ctx)) != cudaSuccess) return e;
  if (ctx->post_on && (e = launch_post_sweep(ctx, 0)) != cudaSuccess) return e;
  k_step_end<<<1, 1, 0, ctx->stream>>>(ctx->clk);
  ctx->launches += 1;
  return cudaGetLastError();
}

// Row bands of imex_gpu_advance_host: more bands shorten the pipeline's fill
// and drain (the first band's upload and the last band's download, which
// nothing overlaps) at a few more launches per band.  At 4096^2 a step from
// and to pinned host memory took 54.0, 49.6 and 47.4 ms with 4, 8 and 16
// bands (63.7 ms as three calls).
#ifndef IMEX_HOST_BANDS
#define IMEX_HOST_BANDS 16
#endif
constexpr int kHostBands = IMEX_HOST_BANDS;

// One driver-loop pass from a host state to a host state, the transfers
// overlapped with the step in row bands.  The bands' host->device copies
// run on the transfer stream; as band b has arrived and been converted,
// the mask of band b-1 and the fluxes of band b-2 run (the mask needs two
// rows of q beyond its band, the fluxes two rows of mask and q).  Stage 2
// up to the Newton passes needs the global dt and runs on the whole grid;
// then each band's assembly and erosion/deposition run and its rows go
// back to the host while the next band computes.  Every cell sees the
// kernels and operations of enqueue_step, in the same order per cell.
template <int NS>
cudaError_t enqueue_host_step_ns(ImexCtx* ctx, const double* q_in, double* q_out) {
  const DevParams& P = ctx->P;
  cudaStream_t st = ctx->stream, cs = ctx->copy_stream;
  const int tiles_x = (P.nx + TX - 1) / TX, tiles_y = (P.ny + TY - 1) / TY;
  const int nb = std::min(kHostBands, tiles_y);
  std::vector<int> tb(nb + 1);
  for (int b = 0; b <= nb; ++b) tb[b] = (int)((long long)b * tiles_y / nb);
  auto r0 = [&](int b) { return tb[b] * TY; };
  auto r1 = [&](int b) { return std::min(tb[b + 1] * TY, P.ny); };
  const size_t row = (size_t)P.nx * P.nv;   // doubles of one AoS grid row
  cudaEvent_t* ev = ctx->band_ev.data();    // [0] start, [1..nb] in, [nb+1..2nb] out
  cudaError_t e;
  // nothing earlier on the stream may still read the staging buffer
  if ((e = cudaEventRecord(ev[0], st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(cs, ev[0], 0)) != cudaSuccess) return e;
  for (int b = 0; b < nb; ++b) {
    const size_t off = (size_t)r0(b) * row, bytes = (size_t)(r1(b) - r0(b)) * row * sizeof(double);
    if ((e = cudaMemcpyAsync(ctx->scratch + off, q_in + off, bytes, cudaMemcpyHostToDevice, cs)) !=
        cudaSuccess)
      return e;
    if ((e = cudaEventRecord(ev[1 + b], cs)) != cudaSuccess) return e;
  }
  k_step_begin<<<1, 1, 0, st>>>(ctx->clk, P.max_dt, 1);
  const size_t smem = sizeof(FluxShared<NS>);
  static std::atomic<unsigned long long> attr_set{0};
  if (attr_needed(attr_set)) {
    for (const void* fn : {(const void*)k_flux_rows<NS>, (const void*)k_flux_tma_rows<NS>}) {
      if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
          cudaSuccess)
        return e;
      if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
        return e;
    }
    attr_done(attr_set);
  }
  int launches = 1;
  auto mask_band = [&](int b) {
    k_mask_rows<<<dim3(tiles_x, tb[b + 1] - tb[b]), 256, 0, st>>>(
        ctx->P, ctx->q, ctx->release, ctx->cellinfo, ctx->clk, ctx->mask, ctx->clk, tb[b]);
    ++launches;
  };
  auto flux_band = [&](int b) {
    const dim3 g(tiles_x, tb[b + 1] - tb[b]);
    if (ctx->q_tmap_ok)
      k_flux_tma_rows<NS><<<g, FLUX_THREADS, smem, st>>>(
          ctx->P, ctx->q_tmap, ctx->q, ctx->mask, ctx->cellinfo, ctx->Bx, ctx->By, ctx->Bxx,
          ctx->Bxy, ctx->Byy, ctx->gc, ctx->dgc, ctx->gcsx, ctx->gcsy, ctx->ring, ctx->clk,
          ctx->X, tb[b]);
    else
      k_flux_rows<NS><<<g, FLUX_THREADS, smem, st>>>(
          ctx->P, ctx->q, ctx->mask, ctx->cellinfo, ctx->Bx, ctx->By, ctx->Bxx, ctx->Bxy,
          ctx->Byy, ctx->gc, ctx->dgc, ctx->gcsx, ctx->gcsy, ctx->ring, ctx->clk, ctx->X, tb[b]);
    ++launches;
  };
  for (int b = 0; b < nb; ++b) {
    if ((e = cudaStreamWaitEvent(st, ev[1 + b], 0)) != cudaSuccess) return e;
    const int rows = r1(b) - r0(b);
    k_aos_to_soa<<<grid_1d((long long)rows * row, 256), 256, 0, st>>>(
        ctx->scratch + (size_t)r0(b) * row, ctx->q + (size_t)r0(b) * P.pitch, P.nv, P.nx, rows,
        P.pitch, P.plane);
    ++launches;
    if (b >= 1) mask_band(b - 1);
    if (b >= 2) flux_band(b - 2);
  }
  mask_band(nb - 1);
  if (nb >= 2) flux_band(nb - 2);
  flux_band(nb - 1);
  k_dt_clip<<<1, 1, 0, st>>>(ctx->clk, 1);
  ++launches;
  // stage 2 through the Newton passes (launch_stage2_ns without assembly)
  const long long ncell = (long long)P.nx * P.ny;
  const int grid = grid_1d(ncell, STAGE2_THREADS);
  const int lgrid = std::min(grid, 148 * IMEX_STAGE2_MINB);
  k_nw_reset<<<1, 1, 0, st>>>(ctx->clk);
  k_stage2_first<NS><<<grid, STAGE2_THREADS, 0, st>>>(ctx->P, ctx->q, ctx->X, ctx->mask, ctx->Bx,
                                                     ctx->By, ctx->Bxx, ctx->Bxy, ctx->Byy,
                                                     ctx->gc, ctx->nw, ctx->clk);
  k_stage2_iter<NS><<<lgrid, STAGE2_THREADS, 0, st>>>(ctx->P, ctx->q, ctx->Bx, ctx->By, ctx->nw,
                                                     ctx->clk, 2);
  k_stage2_iter<NS><<<lgrid, STAGE2_THREADS, 0, st>>>(ctx->P, ctx->q, ctx->Bx, ctx->By, ctx->nw,
                                                     ctx->clk, 3);
  k_stage2_tail<NS><<<lgrid, STAGE2_THREADS, 0, st>>>(ctx->P, ctx->q, ctx->Bx, ctx->By, ctx->nw,
                                                     ctx->clk);
  launches += 5;
  const bool ero = erosion_active(ctx);
  for (int b = 0; b < nb; ++b) {
    const int k0 = r0(b), k1 = r1(b), rows = k1 - k0;
    k_stage2_post_rows<NS><<<grid_1d((long long)rows * P.nx, STAGE2_THREADS), STAGE2_THREADS, 0,
                             st>>>(ctx->P, ctx->q, ctx->mask, ctx->cellinfo, ctx->nw, ctx->clk, k0,
                                   k1);
    ++launches;
    if (ero) {
      k_erosion_rows<NS><<<grid_1d((long long)rows * P.nx, 128), 128, 0, st>>>(
          ctx->P, ctx->q, ctx->mask, ctx->Bx, ctx->By, ctx->erodible, ctx->deposit, ctx->erosion,
          ctx->Bcent, ctx->clk, k0, k1);
      ++launches;
    }
    if (b == nb - 1) {
      k_step_end<<<1, 1, 0, st>>>(ctx->clk);
      ++launches;
    }
    k_soa_to_aos<<<grid_1d((long long)rows * row, 256), 256, 0, st>>>(
        ctx->q + (size_t)k0 * P.pitch, ctx->scratch + (size_t)k0 * row, P.nv, P.nx, rows, P.pitch,
        P.plane);
    ++launches;
    if ((e = cudaEventRecord(ev[1 + nb + b], st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(cs, ev[1 + nb + b], 0)) != cudaSuccess) return e;
    const size_t off = (size_t)k0 * row;
    if ((e = cudaMemcpyAsync(q_out + off, ctx->scratch + off, (size_t)rows * row * sizeof(double),
                             cudaMemcpyDeviceToHost, cs)) != cudaSuccess)
      return e;
  }
  ctx->launches += launches;
  return cudaGetLastError();
}

cudaError_t enqueue_host_step(ImexCtx* ctx, const double* q_in, double* q_out) {
  switch (ctx->ns) {
    case 1: return enqueue_host_step_ns<1>(ctx, q_in, q_out);
    case 2: return enqueue_host_step_ns<2>(ctx, q_in, q_out);
    case 3: return enqueue_host_step_ns<3>(ctx, q_in, q_out);
    default: return enqueue_host_step_ns<4>(ctx, q_in, q_out);
  }
}

int validate(const ImexParams* p, std::string& why) {
  if (p->abi_version != IMEX_ABI_VERSION) { why = "abi_version mismatch"; return IMEX_EINVAL; }
  if (p->nx < 1 || p->ny < 1) { why = "nx and ny must be at least 1"; return IMEX_EINVAL; }
  if (p->n_solid < 1 || p->n_solid > IMEX_MAX_SOLID) { why = "n_solid out of range"; return IMEX_EINVAL; }
  if (p->n_rk != 2) { why = "only the n_RK=2 IMEX tableau is implemented"; return IMEX_EUNSUPPORTED; }
  if (!p->gas_flag || p->liquid_flag) { why = "only a gas carrier phase is implemented"; return IMEX_EUNSUPPORTED; }
  if (p->lateral_source_flag || p->bottom_radial_source_flag) { why = "lateral / bottom sources are not implemented"; return IMEX_EUNSUPPORTED; }
  if (p->rheology_flag && p->rheology_model != 0 && p->rheology_model != 1 && p->rheology_model != 6) {
    why = "rheology models other than 1 (Voellmy-Salm) and 6 (quadratic) are not implemented";
    return IMEX_EUNSUPPORTED;
  }
  const int nv = 4 + p->n_solid;
  for (int i = 0; i < nv + 2; ++i)
    if (p->limiter[i] < 0 || p->limiter[i] > 7) { why = "limiter out of range 0..7"; return IMEX_EINVAL; }
  for (int i = 0; i < nv; ++i) {
    const ImexBC* b[4] = {&p->bcW[i], &p->bcE[i], &p->bcS[i], &p->bcN[i]};
    for (auto* x : b)
      if (x->flag < 0 || x->flag > 2) { why = "boundary flag out of range 0..2"; return IMEX_EINVAL; }
  }
  if (!(p->cell_size > 0.0)) { why = "cell_size must be positive"; return IMEX_EINVAL; }
  if (p->topo_change_flag && (p->nx < 5 || p->ny < 5)) {
    why = "topography update needs at least 5 cells per direction";
    return IMEX_EUNSUPPORTED;
  }
  return IMEX_OK;
}

}  // namespace

namespace {
__global__ void k_point_eval(int fn, long long n, const double* __restrict__ a,
                             const double* __restrict__ b, const double* __restrict__ c,
                             const double* __restrict__ d, double g, double* __restrict__ out) {
  DevParams P;
  P.grav = g;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (fn == 0)   ? ipow(a[i], b[i])
             : (fn == 1) ? settling_velocity(P, a[i], b[i], c[i], d[i])
             : (fn == 2) ? minmod_uniform(a[i], b[i], c[i], d[i], 0.0, d[i], 2.0 * d[i], 1.0)
             : (fn == 3) ? limit(a[i], b[i], c[i], 0.0, d[i], 2.0 * d[i], (int)g, 1.0)
                         : (rel_change_below(a[i], b[i], c[i]) ? 1.0 : 0.0);
}
}  // namespace

// ====================================================================== ABI
extern "C" {

int imex_gpu_point_eval(int fn, long long n, const double* a, const double* b, const double* c,
                        const double* d, double g, double* out) {
  if (fn < 0 || fn > 4 || n < 0 || !a || !b || !out || (fn >= 1 && (!c || !d)))
    return IMEX_EINVAL;
  if (n == 0) return IMEX_OK;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IMEX_ENODEVICE;
  const size_t bytes = (size_t)n * sizeof(double);
  double* buf = nullptr;
  if (cudaMalloc(&buf, 5 * bytes) != cudaSuccess) return IMEX_ENOMEM;
  double *da = buf, *db = buf + n, *dc = buf + 2 * n, *dd = buf + 3 * n, *dout = buf + 4 * n;
  cudaError_t e = cudaMemcpy(da, a, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(db, b, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && fn >= 1) e = cudaMemcpy(dc, c, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && fn >= 1) e = cudaMemcpy(dd, d, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    k_point_eval<<<grid, 256>>>(fn, n, da, db, dc, dd, g, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, bytes, cudaMemcpyDeviceToHost);
  cudaFree(buf);
  return e == cudaSuccess ? IMEX_OK : IMEX_ECUDA;
}

const char* imex_gpu_build_info(void) {
#ifdef IMEX_FMAD
  return "imex_gpu sm_100a fmad=true prec-div prec-sqrt abi=1";
#else
  return "imex_gpu sm_100a fmad=false prec-div prec-sqrt abi=1";
#endif
}

const char* imex_gpu_last_error(ImexCtx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int imex_gpu_create(const ImexParams* p, const ImexStatic* s, int device, ImexCtx** out) {
  if (!p || !s || !out) return IMEX_EINVAL;
  *out = nullptr;
  std::string why;
  int v = validate(p, why);
  if (v != IMEX_OK) {
    fprintf(stderr, "imex_gpu_create: %s\n", why.c_str());
    return v;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return IMEX_ENODEVICE;
  ImexCtx* ctx = new ImexCtx();
  if (device >= 0) {
    CK(cudaSetDevice(device));
    ctx->device = device;
  } else {
    CK(cudaGetDevice(&ctx->device));
  }
  CK(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
  ctx->stream = ctx->own_stream;
  ctx->host_params = *p;
  ctx->ns = p->n_solid;
  DevParams& P = ctx->P;
  P.nx = p->nx;
  P.ny = p->ny;
  P.ns = p->n_solid;
  P.nv = 4 + P.ns;
  P.np = P.nv + 2;
  P.pitch = round_up(P.nx, 16);
  P.plane = P.pitch * P.ny;
  P.x0 = p->x0;
  P.y0 = p->y0;
  // init_grid, src/geometry_2d.f90:250-266: a direction of one cell has
  // spacing 1
  P.dx = (P.nx > 1) ? p->cell_size : 1.0;
  P.dy = (P.ny > 1) ? p->cell_size : 1.0;
  P.dx2 = P.dx / 2.0;
  P.dy2 = P.dy / 2.0;
  P.one_by_dx = 1.0 / P.dx;
  P.one_by_dy = 1.0 / P.dy;
  P.eps_sing = p->eps_sing;
  P.eps_sing4 = (p->eps_sing * p->eps_sing) * (p->eps_sing * p->eps_sing);
  P.hstep = (double)P.nv * EPS;  // src/solver_2d.f90:273
  P.one_by_h = 1.0 / P.hstep;
  P.cfl = p->cfl;
  P.max_dt = p->max_dt;
  P.reconstr_coeff = p->reconstr_coeff;
  P.theta = p->theta;
  for (int i = 0; i < P.nv + 2; ++i) P.limiter[i] = p->limiter[i];
  for (int i = 0; i < P.nv; ++i) {
    P.bcW_flag[i] = p->bcW[i].flag;
    P.bcE_flag[i] = p->bcE[i].flag;
    P.bcS_flag[i] = p->bcS[i].flag;
    P.bcN_flag[i] = p->bcN[i].flag;
    P.bcW_val[i] = p->bcW[i].value;
    P.bcE_val[i] = p->bcE[i].value;
    P.bcS_val[i] = p->bcS[i].value;
    P.bcN_val[i] = p->bcN[i].value;
  }
  P.energy_flag = p->energy_flag;
  P.alpha_flag = p->alpha_flag;
  P.rheology_flag = p->rheology_flag && p->rheology_model != 0;
  P.rheology_model = p->rheology_model;
  P.slope_correction_flag = p->slope_correction_flag;
  P.curvature_term_flag = p->curvature_term_flag;
  P.radial_source_flag = p->radial_source_flag;
  P.settling_flag = p->settling_flag;
  P.entrainment_flag = p->entrainment_flag;
  P.erodible_deposit_flag = p->erodible_deposit_flag;
  P.topo_change_flag = p->topo_change_flag;
  P.grav = p->grav;
  P.T_ambient = p->T_ambient;
  P.pres = p->pres;
  P.inv_pres = 1.0 / p->pres;  // src/inpout_2d.f90:1330
  P.sp_heat_a = p->sp_heat_a;
  P.sp_gas_const_a = p->sp_gas_const_a;
  P.kin_visc_c = p->kin_visc_c;
  P.rho_a_amb = p->pres / (p->sp_gas_const_a * p->T_ambient);  // src/inpout_2d.f90:1353
  for (int i = 0; i < P.ns; ++i) {
    P.rho_s[i] = p->rho_s[i];
    P.inv_rho_s[i] = 1.0 / p->rho_s[i];
    P.diam_s[i] = p->diam_s[i];
    P.sp_heat_s[i] = p->sp_heat_s[i];
    P.alphas_source[i] = p->alphas_source[i];
    P.erodible_fract[i] = p->erodible_fract[i];
  }
  P.mu = p->mu;
  P.xi = p->xi;
  P.friction_factor = p->friction_factor;
  P.maximum_solid_packing = p->maximum_solid_packing;
  P.h_source = p->h_source;
  P.vel_source = p->vel_source;
  P.T_source = p->T_source;
  for (int i = 0; i < 4; ++i) P.time_param[i] = p->time_param[i];
  P.erosion_coeff = p->erosion_coeff;
  P.erodible_porosity = p->erodible_porosity;
  P.T_erodible = p->T_erodible;
  P.alphastot_min = p->alphastot_min;
  P.rho_c_sub = p->rho_c_sub;
  P.coeff_porosity = p->coeff_porosity;

  const int nx = P.nx, ny = P.ny, nv = P.nv;
  const size_t N = (size_t)nx * ny;
  if (!s->B_prime_x_geom || !s->B_prime_y_geom) {
    delete ctx;
    return IMEX_EINVAL;
  }
  if (P.slope_correction_flag && (!s->grav_coeff || !s->grav_coeff_stag_x || !s->grav_coeff_stag_y || !s->d_grav_coeff_dx)) {
    delete ctx;
    return IMEX_EINVAL;
  }
  if (P.curvature_term_flag && (!s->B_second_xx_geom || !s->B_second_xy_geom || !s->B_second_yy_geom)) {
    delete ctx;
    return IMEX_EINVAL;
  }
  // cell info: source_cell + inlet flags + B_nodata
  std::vector<uint8_t> info(N, 0);
  std::vector<RingCell> ring;
  bool any_info = false;
  if (P.radial_source_flag) {
    if (!s->source_cell || !s->sourceE || !s->sourceW || !s->sourceS || !s->sourceN) {
      delete ctx;
      return IMEX_EINVAL;
    }
    for (size_t c = 0; c < N; ++c) {
      int sc = s->source_cell[c];
      uint8_t b = (uint8_t)(sc & 3);
      if (s->sourceE[c]) b |= CI_E;
      if (s->sourceW[c]) b |= CI_W;
      if (s->sourceS[c]) b |= CI_S;
      if (s->sourceN[c]) b |= CI_N;
      info[c] = b;
      if (sc == 2) {
        RingCell r{};
        r.idx = (int64_t)c;
        const double* vx[4] = {s->sourceE_vect_x, s->sourceW_vect_x, s->sourceS_vect_x, s->sourceN_vect_x};
        const double* vy[4] = {s->sourceE_vect_y, s->sourceW_vect_y, s->sourceS_vect_y, s->sourceN_vect_y};
        for (int w = 0; w < 4; ++w) {
          r.vx[w] = vx[w] ? vx[w][c] : 0.0;
          r.vy[w] = vy[w] ? vy[w][c] : 0.0;
        }
        ring.push_back(r);
      }
      if (b) any_info = true;
    }
  }
  if (s->B_nodata)
    for (size_t c = 0; c < N; ++c)
      if (s->B_nodata[c]) {
        info[c] |= CI_NODATA;
        any_info = true;
      }
  P.has_cellinfo = any_info ? 1 : 0;
  P.n_ring = (int)ring.size();
  bool has_rel = false;
  if (s->solve_mask_time)
    for (size_t c = 0; c < N; ++c)
      if (s->solve_mask_time[c] != 0.0) { has_rel = true; break; }
  P.has_release_time = has_rel ? 1 : 0;
  ctx->exchange = erosion_active(ctx);
  P.has_exchange = ctx->exchange ? 1 : 0;
  if (ctx->exchange && (!s->erodible || !s->deposit || !s->erosion)) {
    delete ctx;
    return IMEX_EINVAL;
  }

  const size_t plane = (size_t)P.plane;
  if (plane > (size_t)UINT32_MAX) {
    delete ctx;
    return IMEX_EUNSUPPORTED;  // stage-2 cell lists hold 32-bit plane indices
  }
  CK(dalloc(&ctx->q, plane * nv));
  ctx->q_tmap_ok = encode_q_map(ctx);
  CK(dalloc(&ctx->X, plane * nv));
  CK(dalloc(&ctx->mask, plane));
  CK(cudaMemset(ctx->q, 0, plane * nv * sizeof(double)));
  CK(cudaMemset(ctx->X, 0, plane * nv * sizeof(double)));
  CK(cudaMemset(ctx->mask, 0, plane));
  CK(dalloc(&ctx->cellinfo, N));
  CK(cudaMemcpy(ctx->cellinfo, info.data(), N, cudaMemcpyHostToDevice));
  CK(dalloc(&ctx->ring, std::max<size_t>(ring.size(), 1)));
  if (!ring.empty()) CK(cudaMemcpy(ctx->ring, ring.data(), ring.size() * sizeof(RingCell), cudaMemcpyHostToDevice));
  CK(dalloc(&ctx->Bx, plane));
  CK(dalloc(&ctx->By, plane));
  CK(upload_plane(ctx, ctx->Bx, s->B_prime_x_geom, 0.0));
  CK(upload_plane(ctx, ctx->By, s->B_prime_y_geom, 0.0));
  if (P.curvature_term_flag) {
    CK(dalloc(&ctx->Bxx, plane));
    CK(dalloc(&ctx->Bxy, plane));
    CK(dalloc(&ctx->Byy, plane));
    CK(upload_plane(ctx, ctx->Bxx, s->B_second_xx_geom, 0.0));
    CK(upload_plane(ctx, ctx->Bxy, s->B_second_xy_geom, 0.0));
    CK(upload_plane(ctx, ctx->Byy, s->B_second_yy_geom, 0.0));
  }
  if (P.topo_change_flag && !P.curvature_term_flag) {
    // the bed-change update writes the second derivatives (grav_coeff's
    // derivative needs them); the step reads them only with curvature on
    CK(dalloc(&ctx->Bxx, plane));
    CK(dalloc(&ctx->Bxy, plane));
    CK(dalloc(&ctx->Byy, plane));
    CK(cudaMemset(ctx->Bxx, 0, plane * sizeof(double)));
    CK(cudaMemset(ctx->Bxy, 0, plane * sizeof(double)));
    CK(cudaMemset(ctx->Byy, 0, plane * sizeof(double)));
  }
  if (P.slope_correction_flag) {
    CK(dalloc(&ctx->gc, plane));
    CK(dalloc(&ctx->dgc, plane));
    CK(upload_plane(ctx, ctx->gc, s->grav_coeff, 1.0));
    CK(upload_plane(ctx, ctx->dgc, s->d_grav_coeff_dx, 0.0));
    CK(dalloc(&ctx->gcsx, (size_t)(nx + 1) * ny));
    CK(dalloc(&ctx->gcsy, (size_t)nx * (ny + 1)));
    CK(cudaMemcpy(ctx->gcsx, s->grav_coeff_stag_x, (size_t)(nx + 1) * ny * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->gcsy, s->grav_coeff_stag_y, (size_t)nx * (ny + 1) * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (has_rel) {
    CK(dalloc(&ctx->release, plane));
    CK(upload_plane(ctx, ctx->release, s->solve_mask_time, 0.0));
  }
  if (!ctx->exchange && !P.topo_change_flag && s->B_cent) {   // for the output writers
    CK(dalloc(&ctx->Bcent, plane));
    CK(upload_plane(ctx, ctx->Bcent, s->B_cent, 0.0));
  }
  if (ctx->exchange || P.topo_change_flag) {
    const int ns = P.ns;
    CK(dalloc(&ctx->erodible, plane * ns));
    CK(dalloc(&ctx->deposit, plane * ns));
    CK(dalloc(&ctx->erosion, plane * ns));
    CK(dalloc(&ctx->Bcent, plane));
    std::vector<double> tmp(N);
    for (int i = 0; i < ns; ++i) {
      for (size_t c = 0; c < N; ++c) tmp[c] = s->erodible ? s->erodible[(size_t)i + ns * c] : 0.0;
      CK(upload_plane(ctx, ctx->erodible + plane * i, tmp.data(), 0.0));
      CK(upload_plane(ctx, ctx->deposit + plane * i, s->deposit ? s->deposit + N * i : nullptr, 0.0));
      CK(upload_plane(ctx, ctx->erosion + plane * i, s->erosion ? s->erosion + N * i : nullptr, 0.0));
    }
    CK(upload_plane(ctx, ctx->Bcent, s->B_cent, 0.0));
  }
  CK(cudaMalloc((void**)&ctx->dP, sizeof(DevParams)));
  CK(cudaMemcpy(ctx->dP, &ctx->P, sizeof(DevParams), cudaMemcpyHostToDevice));
  CK(cudaMalloc((void**)&ctx->clk, sizeof(DevClock)));
  CK(cudaMallocHost((void**)&ctx->clk_host, sizeof(DevClock)));
  std::memset(ctx->clk_host, 0, sizeof(DevClock));
  ctx->clk_host->first_error = ~0ULL;
  ctx->clk_host->t_end = 1e300;
  ctx->clk_host->t_output = -1.0;
  ctx->clk_host->dt_old = ctx->clk_host->dt_old_old = p->max_dt;
  CK(cudaMemcpy(ctx->clk, ctx->clk_host, sizeof(DevClock), cudaMemcpyHostToDevice));
  ctx->scratch_bytes = N * (size_t)(nv + 2) * sizeof(double);
  CK(cudaMalloc((void**)&ctx->scratch, ctx->scratch_bytes));
  // stage-2 Newton state: q_si, Rj, iterate, residual (nv planes each), |r|^2/2
  CK(dalloc(&ctx->nw_buf, plane * (4 * (size_t)nv + 1)));
  CK(dalloc(&ctx->nw.status, plane));
  CK(dalloc(&ctx->nw_lists, plane * 3));
  ctx->nw.qsi = ctx->nw_buf;
  ctx->nw.Rj = ctx->nw_buf + plane * nv;
  ctx->nw.x = ctx->nw_buf + plane * nv * 2;
  ctx->nw.rt = ctx->nw_buf + plane * nv * 3;
  ctx->nw.sf = ctx->nw_buf + plane * nv * 4;
  for (int i = 0; i < 3; ++i) ctx->nw.list[i] = ctx->nw_lists + plane * i;
  CK(cudaDeviceSynchronize());
  *out = ctx;
  return IMEX_OK;
}

int imex_gpu_destroy(ImexCtx* ctx) {
  if (!ctx) return IMEX_EINVAL;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->out_thread.joinable()) ctx->out_thread.join();
  if (ctx->out_dev) cudaFree(ctx->out_dev);
  if (ctx->out_host) cudaFreeHost(ctx->out_host);
  if (ctx->out_ev) cudaEventDestroy(ctx->out_ev);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  void* bufs[] = {ctx->q, ctx->X, ctx->mask, ctx->cellinfo, ctx->Bx, ctx->By, ctx->Bxx, ctx->Bxy,
                  ctx->Byy, ctx->gc, ctx->dgc, ctx->gcsx, ctx->gcsy, ctx->release, ctx->erodible,
                  ctx->deposit, ctx->erosion, ctx->Bcent, ctx->ring, ctx->clk, ctx->scratch, ctx->dP,
                  ctx->nw_buf, ctx->nw.status, ctx->nw_lists, ctx->post_buf, ctx->post_vuln,
                  ctx->post_diag, ctx->nw_wlist, ctx->nw_feat, ctx->nw_guess, ctx->h_x, ctx->h_y};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (ctx->clk_host) cudaFreeHost(ctx->clk_host);
  for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->band_ev) cudaEventDestroy(e);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return IMEX_OK;
}

static int push_time(ImexCtx* ctx, double t, const double* dt) {
  // clock fields live on the device; patch t (and dt) with small copies
  CK(cudaMemcpyAsync(&ctx->clk->t, &t, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (dt) CK(cudaMemcpyAsync(&ctx->clk->dt, dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

int imex_gpu_set_state(ImexCtx* ctx, const double* q, double t) {
  if (!ctx || !q) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  const DevParams& P = ctx->P;
  const size_t n = (size_t)P.nx * P.ny * P.nv;
  CK(cudaMemcpyAsync(ctx->scratch, q, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  k_aos_to_soa<<<grid_1d((long long)n, 256), 256, 0, ctx->stream>>>(ctx->scratch, ctx->q, P.nv, P.nx, P.ny, P.pitch, P.plane);
  ctx->launches += 1;
  CK(cudaGetLastError());
  ctx->x_valid = false;
  int r = push_time(ctx, t, nullptr);
  if (r) return r;
  int64_t ncells = 0;
  return imex_gpu_check_solve(ctx, t, 1, &ncells);
}

int imex_gpu_get_state(ImexCtx* ctx, double* q, double* qp) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  const DevParams& P = ctx->P;
  const size_t N = (size_t)P.nx * P.ny;
  if (q) {
    k_soa_to_aos<<<grid_1d((long long)N * P.nv, 256), 256, 0, ctx->stream>>>(ctx->q, ctx->scratch, P.nv, P.nx, P.ny, P.pitch, P.plane);
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(q, ctx->scratch, N * P.nv * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  if (qp) {
    switch (ctx->ns) {
      case 1: k_qp_out<1><<<grid_1d((long long)N, 128), 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->scratch, ctx->cellinfo); break;
      case 2: k_qp_out<2><<<grid_1d((long long)N, 128), 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->scratch, ctx->cellinfo); break;
      case 3: k_qp_out<3><<<grid_1d((long long)N, 128), 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->scratch, ctx->cellinfo); break;
      default: k_qp_out<4><<<grid_1d((long long)N, 128), 128, 0, ctx->stream>>>(ctx->P, ctx->q, ctx->scratch, ctx->cellinfo); break;
    }
    ctx->launches += 1;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(qp, ctx->scratch, N * P.np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return IMEX_OK;
}

int imex_gpu_get_exchange(ImexCtx* ctx, double* erodible, double* deposit, double* erosion,
                          double* B_cent) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  const DevParams& P = ctx->P;
  const int nx = P.nx, ny = P.ny, ns = P.ns;
  const size_t N = (size_t)nx * ny, plane = (size_t)P.plane;
  if (!ctx->erodible) return (erodible || deposit || erosion || B_cent) ? IMEX_EINVAL : IMEX_OK;
  std::vector<double> h(plane);
  auto fetch = [&](const double* dsrc, double* out, size_t out_stride, size_t out_off, size_t elem_stride) -> int {
    CK(cudaMemcpy(h.data(), dsrc, plane * sizeof(double), cudaMemcpyDeviceToHost));
    for (int k = 0; k < ny; ++k)
      for (int j = 0; j < nx; ++j)
        out[out_off + ((size_t)j + (size_t)nx * k) * elem_stride] = h[(size_t)k * P.pitch + j];
    (void)out_stride;
    return IMEX_OK;
  };
  for (int i = 0; i < ns; ++i) {
    if (erodible && fetch(ctx->erodible + plane * i, erodible, 0, (size_t)i, (size_t)ns)) return IMEX_ECUDA;
    if (deposit && fetch(ctx->deposit + plane * i, deposit, 0, N * i, 1)) return IMEX_ECUDA;
    if (erosion && fetch(ctx->erosion + plane * i, erosion, 0, N * i, 1)) return IMEX_ECUDA;
  }
  if (B_cent && fetch(ctx->Bcent, B_cent, 0, 0, 1)) return IMEX_ECUDA;
  return IMEX_OK;
}

int imex_gpu_check_solve(ImexCtx* ctx, double t, int solve_all, int64_t* n_solve_cells) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  int r = push_time(ctx, t, nullptr);
  if (r) return r;
  const unsigned long long zero = 0;
  CK(cudaMemcpyAsync(&ctx->clk->solve_cells, &zero, sizeof(unsigned long long), cudaMemcpyHostToDevice, ctx->stream));
  CK(launch_mask(ctx, solve_all ? 1 : 0));
  ctx->x_valid = false;
  unsigned long long cnt = 0;
  CK(cudaMemcpyAsync(&cnt, &ctx->clk->solve_cells, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (n_solve_cells) *n_solve_cells = (int64_t)cnt;
  return IMEX_OK;
}

int imex_gpu_timestep(ImexCtx* ctx, double* dt) {
  if (!ctx || !dt) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  k_step_begin<<<1, 1, 0, ctx->stream>>>(ctx->clk, ctx->P.max_dt, 0);
  ctx->launches += 1;
  if (ctx->P.cfl != -1.0) {
    CK(launch_flux(ctx));
    ctx->x_valid = true;
  }
  k_dt_clip<<<1, 1, 0, ctx->stream>>>(ctx->clk, 0);
  ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dt, &ctx->clk->dt, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

static int collect_errors(ImexCtx* ctx) {
  unsigned int em = 0;
  CK(cudaMemcpyAsync(&em, &ctx->clk->error_mask, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  uint32_t fresh = em & ~ctx->error_mask_acc;
  ctx->error_mask_acc |= em;
  if (!fresh) return IMEX_OK;
  for (int code = 1; code <= 7; ++code)
    if (fresh & (1u << code)) return code;
  return IMEX_OK;
}

int imex_gpu_rk_step(ImexCtx* ctx, double t, double dt) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  int r = push_time(ctx, t, &dt);
  if (r) return r;
  if (!ctx->x_valid) CK(launch_flux(ctx));
  CK(launch_stage2(ctx));
  ctx->x_valid = false;
  return collect_errors(ctx);
}

int imex_gpu_erosion_deposition(ImexCtx* ctx, double dt) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->exchange) return IMEX_OK;  // src/solver_2d.f90:2424-2425
  CK(cudaMemcpyAsync(&ctx->clk->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(launch_erosion(ctx));
  ctx->x_valid = false;
  return collect_errors(ctx);
}

int imex_gpu_get_masks(ImexCtx* ctx, int8_t* solve_mask, int8_t* mask_x, int8_t* mask_y) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  const DevParams& P = ctx->P;
  const int nx = P.nx, ny = P.ny;
  CK(cudaStreamSynchronize(ctx->stream));
  if (solve_mask) {
    std::vector<uint8_t> m((size_t)P.plane);
    CK(cudaMemcpy(m.data(), ctx->mask, m.size(), cudaMemcpyDeviceToHost));
    for (int k = 0; k < ny; ++k)
      for (int j = 0; j < nx; ++j) solve_mask[(size_t)j + (size_t)nx * k] = (int8_t)m[(size_t)k * P.pitch + j];
  }
  if (mask_x || mask_y) {
    size_t nX = (size_t)(nx + 1) * ny, nY = (size_t)nx * (ny + 1);
    int8_t* d = reinterpret_cast<int8_t*>(ctx->scratch);
    k_masks_xy<<<grid_1d((long long)(nX + nY), 256), 256, 0, ctx->stream>>>(ctx->P, ctx->mask, d, d + nX);
    ctx->launches += 1;
    CK(cudaGetLastError());
    if (mask_x) CK(cudaMemcpyAsync(mask_x, d, nX, cudaMemcpyDeviceToHost, ctx->stream));
    if (mask_y) CK(cudaMemcpyAsync(mask_y, d + nX, nY, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  return IMEX_OK;
}

int imex_gpu_set_clock(ImexCtx* ctx, double t, double dt0, double t_end, double t_output) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(ctx->clk_host, ctx->clk, sizeof(DevClock), cudaMemcpyDeviceToHost));
  ctx->clk_host->t = t;
  ctx->clk_host->dt_old = dt0;
  ctx->clk_host->dt_old_old = dt0;
  ctx->clk_host->t_end = t_end;
  ctx->clk_host->t_output = t_output;
  CK(cudaMemcpy(ctx->clk, ctx->clk_host, sizeof(DevClock), cudaMemcpyHostToDevice));
  ctx->x_valid = false;
  return IMEX_OK;
}

int imex_gpu_advance(ImexCtx* ctx, int n_steps, int use_graph, double* t) {
  if (!ctx || n_steps < 0) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  if (use_graph) {
    if (!ctx->graph_exec) {
      int64_t l0 = ctx->launches;
      CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue_step(ctx);
      cudaGraph_t g = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
      if (e != cudaSuccess) return fail(ctx, IMEX_ECUDA, cudaGetErrorString(e));
      if (e2 != cudaSuccess) return fail(ctx, IMEX_ECUDA, cudaGetErrorString(e2));
      ctx->graph = g;
      CK(cudaGraphInstantiate(&ctx->graph_exec, g, 0));
      ctx->graph_launches = ctx->launches - l0;
      ctx->launches = l0;
    }
    for (int s = 0; s < n_steps; ++s) {
      CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
      ctx->launches += ctx->graph_launches;
    }
  } else {
    for (int s = 0; s < n_steps; ++s) {
      cudaError_t e = enqueue_step(ctx);
      if (e != cudaSuccess) return fail(ctx, IMEX_ECUDA, cudaGetErrorString(e));
    }
  }
  ctx->x_valid = false;
  if (t) {
    CK(cudaMemcpyAsync(t, &ctx->clk->t, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  }
  int r = collect_errors(ctx);
  return r;
}

int imex_gpu_advance_host(ImexCtx* ctx, const double* q_in, double t, double* q_out,
                          double* t_out) {
  if (!ctx || !q_in || !q_out) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  if (ctx->nw.warm || ctx->nw.harvest || ctx->P.topo_change_flag || ctx->post_on || ctx->prof) {
    // options the banded step leaves out: the three calls in sequence
    int r = imex_gpu_set_state(ctx, q_in, t);
    if (r) return r;
    const int ra = imex_gpu_advance(ctx, 1, 0, t_out);
    if (ra >= IMEX_ETIMEOUT) return ra;
    r = imex_gpu_get_state(ctx, q_out, nullptr);
    return r ? r : ra;
  }
  if (!ctx->copy_stream) CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  while (ctx->band_ev.size() < (size_t)(2 * kHostBands + 1)) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ctx->band_ev.push_back(ev);
  }
  int r = push_time(ctx, t, nullptr);
  if (r) return r;
  ctx->x_valid = false;
  cudaError_t e = enqueue_host_step(ctx, q_in, q_out);
  if (e != cudaSuccess) return fail(ctx, IMEX_ECUDA, cudaGetErrorString(e));
  CK(cudaStreamSynchronize(ctx->copy_stream));
  if (t_out)
    CK(cudaMemcpyAsync(t_out, &ctx->clk->t, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  return collect_errors(ctx);
}

int imex_gpu_stats(ImexCtx* ctx, ImexStats* st, int reset_errors) {
  if (!ctx || !st) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(ctx->clk_host, ctx->clk, sizeof(DevClock), cudaMemcpyDeviceToHost));
  const DevClock& c = *ctx->clk_host;
  std::memset(st, 0, sizeof(*st));
  st->solve_cells = c.solve_cells;
  st->newton_cells = c.newton_cells;
  st->newton_iters = c.newton_iters;
  st->lnsrch_trials = c.lnsrch_trials;
  st->newton_maxit_cells = c.newton_maxit;
  for (int b = 0; b < 16; ++b) st->newton_hist[b] = c.hist[b];
  st->error_mask = c.error_mask;
  if (c.first_error != ~0ULL) {
    long long cell = (long long)(c.first_error >> 8);
    st->first_error_code = (int)(c.first_error & 0xff);
    st->first_error_j = (int32_t)(cell % ctx->P.nx) + 1;
    st->first_error_k = (int32_t)(cell / ctx->P.nx) + 1;
  }
  st->dt = c.dt;
  st->t = c.t;
  st->steps = c.steps;
  st->kernel_launches = ctx->launches;
  st->warm_fallback_cells = (int64_t)c.warm_fallback;
  if (reset_errors) {
    ctx->clk_host->error_mask = 0;
    ctx->clk_host->first_error = ~0ULL;
    CK(cudaMemcpy(&ctx->clk->error_mask, &ctx->clk_host->error_mask, sizeof(unsigned int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&ctx->clk->first_error, &ctx->clk_host->first_error, sizeof(unsigned long long), cudaMemcpyHostToDevice));
    ctx->error_mask_acc = 0;
  }
  return IMEX_OK;
}

int imex_gpu_sync(ImexCtx* ctx) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

int imex_gpu_set_stream(ImexCtx* ctx, void* stream) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own_stream;
  if (s != ctx->stream) {
    // a captured graph is bound to nothing stream-specific, but keep the
    // capture on the stream it will be replayed on
    if (ctx->graph_exec) {
      cudaGraphExecDestroy(ctx->graph_exec);
      ctx->graph_exec = nullptr;
    }
    if (ctx->graph) {
      cudaGraphDestroy(ctx->graph);
      ctx->graph = nullptr;
    }
  }
  ctx->stream = s;
  return IMEX_OK;
}

int imex_gpu_profile(ImexCtx* ctx, int enable) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->prof = enable != 0;
  ctx->ev_pending.clear();
  ctx->ev_used = 0;
  return IMEX_OK;
}

int imex_gpu_kernel_times(ImexCtx* ctx, double* total_ms, int64_t* launches, int n_kernels) {
  if (!ctx || !total_ms || !launches || n_kernels < KID_N) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n_kernels; ++i) {
    total_ms[i] = 0.0;
    launches[i] = 0;
  }
  for (auto& pe : ctx->ev_pending) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, pe.second.first, pe.second.second));
    total_ms[pe.first] += ms;
    launches[pe.first] += 1;
  }
  ctx->ev_pending.clear();
  ctx->ev_used = 0;
  return IMEX_OK;
}

int imex_gpu_measure_fp64_peak(int device, double* gflops) {
  ImexCtx* ctx = nullptr;
  if (!gflops) return IMEX_EINVAL;
  if (device >= 0) CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaGetDeviceProperties(&prop, dev));
  double* out = nullptr;
  CK(cudaMalloc((void**)&out, sizeof(double)));
  const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 1 << 14;
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  k_fp64_probe<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);
  CK(cudaDeviceSynchronize());
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    CK(cudaEventRecord(a));
    k_fp64_probe<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    CK(cudaEventRecord(b));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, ms);
  }
  double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
  *gflops = flops / (best * 1e-3) / 1e9;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  return IMEX_OK;
}

int imex_gpu_device_state(ImexCtx* ctx, double** q_dev, int64_t* pitch) {
  if (!ctx) return IMEX_EINVAL;
  if (q_dev) *q_dev = ctx->q;
  if (pitch) *pitch = ctx->P.pitch;
  return IMEX_OK;
}

}  // extern "C"

// ============================================================ post step
extern "C" {

int imex_gpu_post_init(ImexCtx* ctx, int n_thickness_levels, const double* thickness_levels,
                       int n_dyn_pres_levels, const double* dyn_pres_levels) {
  if (!ctx) return IMEX_EINVAL;
  int nt = std::max(n_thickness_levels, 0), np = std::max(n_dyn_pres_levels, 0);
  if (nt > POST_MAX_LEVELS || np > POST_MAX_LEVELS || (nt && !thickness_levels) ||
      (np && !dyn_pres_levels))
    return fail(ctx, IMEX_EINVAL, "imex_gpu_post_init: at most 10 levels of each kind");
  PostLevels L{};
  for (int i = 0; i < nt; ++i) L.thk[i] = thickness_levels[i];
  for (int i = 0; i < np; ++i) L.pdyn[i] = dyn_pres_levels[i];
  for (int i = 0; i < nt; ++i)
    if (!(L.thk[i] >= 0.0)) return fail(ctx, IMEX_EINVAL, "imex_gpu_post_init: negative thickness level");
  for (int i = 0; i < np; ++i)
    if (!(L.pdyn[i] >= 0.0)) return fail(ctx, IMEX_EINVAL, "imex_gpu_post_init: negative pressure level");
  // one kind given alone: the other is a single level 0 (src/inpout_2d.f90:3630-3682)
  if (nt > 0 && np == 0) { np = 1; L.pdyn[0] = 0.0; }
  if (np > 0 && nt == 0) { nt = 1; L.thk[0] = 0.0; }
  L.n_thk = nt;
  L.n_pdyn = np;
  L.n_words = (nt * np + 31) / 32;
  CK(cudaSetDevice(ctx->device));
  const size_t plane = (size_t)ctx->P.plane;
  if (!ctx->post_buf) {
    CK(dalloc(&ctx->post_buf, plane * 4));
    CK(dalloc(&ctx->post_diag, 4 + 4 * (size_t)DIAG_BLOCKS));
  }
  if (ctx->post_vuln) {
    cudaFree(ctx->post_vuln);
    ctx->post_vuln = nullptr;
  }
  if (L.n_words) CK(dalloc(&ctx->post_vuln, plane * L.n_words));
  ctx->post.qp_h = ctx->post_buf;
  ctx->post.hmax = ctx->post_buf + plane;
  ctx->post.pdynmax = ctx->post_buf + 2 * plane;
  ctx->post.mvmax = ctx->post_buf + 3 * plane;
  ctx->post.vuln = ctx->post_vuln;
  ctx->post_levels = L;
  CK(cudaMemsetAsync(ctx->post_buf, 0, plane * 4 * sizeof(double), ctx->stream));
  if (ctx->post_vuln)
    CK(cudaMemsetAsync(ctx->post_vuln, 0, plane * L.n_words * sizeof(uint32_t), ctx->stream));
  CK(launch_post_sweep(ctx, 1));
  // a captured step does not hold the sweep yet
  if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
  ctx->post_on = true;
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

int imex_gpu_topography_reconstruction(ImexCtx* ctx) {
  if (!ctx) return IMEX_EINVAL;
  if (!ctx->Bcent) return fail(ctx, IMEX_EINVAL, "topography update: no B_cent plane");
  CK(cudaSetDevice(ctx->device));
  CK(launch_topo(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

int imex_gpu_post_diag(ImexCtx* ctx, ImexPostDiag* diag) {
  if (!ctx || !diag) return IMEX_EINVAL;
  if (!ctx->post_on) return fail(ctx, IMEX_EINVAL, "imex_gpu_post_diag: call imex_gpu_post_init first");
  CK(cudaSetDevice(ctx->device));
  CK(launch_post_diag(ctx));
  double out[4];
  CK(cudaMemcpyAsync(out, ctx->post_diag, sizeof(out), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  const double cell = ctx->P.dx * ctx->P.dy;
  diag->mass = cell * out[0];
  diag->volume = cell * out[1];
  diag->area = cell * out[2];
  diag->solid_mass = cell * out[3];
  return IMEX_OK;
}

int imex_gpu_post_step(ImexCtx* ctx, ImexPostDiag* diag) {
  if (!ctx) return IMEX_EINVAL;
  if (!ctx->post_on) return fail(ctx, IMEX_EINVAL, "imex_gpu_post_step: call imex_gpu_post_init first");
  CK(cudaSetDevice(ctx->device));
  CK(launch_post_sweep(ctx, 0));
  if (diag) return imex_gpu_post_diag(ctx, diag);
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

int imex_gpu_get_post(ImexCtx* ctx, double* hmax, double* pdynmax, double* mod_vel_max,
                      int8_t* vuln_table, int* n_table) {
  if (!ctx) return IMEX_EINVAL;
  if (!ctx->post_on) return fail(ctx, IMEX_EINVAL, "imex_gpu_get_post: call imex_gpu_post_init first");
  CK(cudaSetDevice(ctx->device));
  const DevParams& P = ctx->P;
  const size_t nx = (size_t)P.nx, ny = (size_t)P.ny, pitch = (size_t)P.pitch;
  double* planes[3] = {hmax, pdynmax, mod_vel_max};
  const double* src[3] = {ctx->post.hmax, ctx->post.pdynmax, ctx->post.mvmax};
  for (int i = 0; i < 3; ++i)
    if (planes[i])
      CK(cudaMemcpy2DAsync(planes[i], nx * sizeof(double), src[i], pitch * sizeof(double),
                           nx * sizeof(double), ny, cudaMemcpyDeviceToHost, ctx->stream));
  const int nt = ctx->post_levels.n_thk * ctx->post_levels.n_pdyn;
  if (n_table) *n_table = nt;
  if (vuln_table && nt) {
    const int nw = ctx->post_levels.n_words;
    std::vector<uint32_t> w(pitch * ny * nw);
    CK(cudaMemcpyAsync(w.data(), ctx->post_vuln, w.size() * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (size_t k = 0; k < ny; ++k)
      for (size_t j = 0; j < nx; ++j)
        for (int i = 0; i < nt; ++i) {
          uint32_t word = w[(size_t)(i >> 5) * pitch * ny + k * pitch + j];
          vuln_table[(size_t)i + (size_t)nt * (j + nx * k)] = (int8_t)((word >> (i & 31)) & 1u);
        }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

}  // extern "C"

// =================================================================== MLP
struct ImexMLP {
  int device = 0;
  float* prm = nullptr;        // FP32 master parameters
  float* grad = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  float* loss = nullptr;       // summed squared error of the last pass
  __nv_bfloat16* bw = nullptr; // BF16 weights
  int64_t adam_t = 0;
  float norm[2 * mlp::IN + 2 * mlp::OUT] = {};  // x mean, x std, y mean, y std
  std::string last_error;
};

namespace {

int mlp_fail(ImexMLP* m, int code, const std::string& msg) {
  if (m) m->last_error = msg;
  return code;
}
#define CKM(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) return mlp_fail(mlp, IMEX_ECUDA, cudaGetErrorString(e_)); \
  } while (0)

uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

int mlp_refresh_bf16(ImexMLP* mlp) {
  mlp::k_mlp_to_bf16<<<(mlp::NBW + 255) / 256, 256>>>(mlp->prm, mlp->bw);
  CKM(cudaGetLastError());
  return IMEX_OK;
}

int mlp_grad_pass(ImexMLP* mlp, const float* x, const float* y, long long n) {
  static std::atomic<unsigned long long> attr{0};
  if (attr_needed(attr)) {
    CKM(cudaFuncSetAttribute(mlp::k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)mlp::SMEM_GRAD));
    attr_done(attr);
  }
  const long long tiles = (n + mlp::SAMPLES - 1) / mlp::SAMPLES;
  const int grid = (int)std::max<long long>(1, std::min<long long>(tiles, 148));
  CKM(cudaMemset(mlp->loss, 0, sizeof(float)));
  mlp::k_mlp_grad<<<grid, 32 * mlp::WARPS, mlp::SMEM_GRAD>>>(
      mlp->bw, mlp->prm, x, y, n, 1.0f / (float)(n * mlp::OUT), mlp->grad, mlp->loss);
  CKM(cudaGetLastError());
  return IMEX_OK;
}

}  // namespace

extern "C" {

int imex_mlp_create(int device, uint64_t seed, ImexMLP** out) {
  if (!out) return IMEX_EINVAL;
  *out = nullptr;
  ImexMLP* mlp = new ImexMLP();
  if (device >= 0) CKM(cudaSetDevice(device));
  CKM(cudaGetDevice(&mlp->device));
  // He-uniform weights on the real rows/columns, zero padding and biases
  std::vector<float> p(mlp::NPARAM, 0.0f);
  uint64_t st = seed;
  auto fill = [&](int off, int rows, int cols, int real_rows, int real_cols) {
    const double a = std::sqrt(6.0 / real_rows);
    for (int r = 0; r < real_rows; ++r)
      for (int c = 0; c < real_cols; ++c) p[off + r * cols + c] = (float)((2.0 * uniform01(st) - 1.0) * a);
    (void)rows;
  };
  fill(mlp::OFF_W0, mlp::IN_P, mlp::HID, mlp::IN, mlp::HID);
  fill(mlp::OFF_W1, mlp::HID, mlp::HID, mlp::HID, mlp::HID);
  fill(mlp::OFF_W2, mlp::HID, mlp::HID, mlp::HID, mlp::HID);
  fill(mlp::OFF_W3, mlp::HID, mlp::OUT_P, mlp::HID, mlp::OUT);
  CKM(cudaMalloc((void**)&mlp->prm, mlp::NPARAM * sizeof(float)));
  CKM(cudaMalloc((void**)&mlp->grad, mlp::NPARAM * sizeof(float)));
  CKM(cudaMalloc((void**)&mlp->m1, mlp::NPARAM * sizeof(float)));
  CKM(cudaMalloc((void**)&mlp->m2, mlp::NPARAM * sizeof(float)));
  CKM(cudaMalloc((void**)&mlp->loss, sizeof(float)));
  CKM(cudaMalloc((void**)&mlp->bw, mlp::NBW * sizeof(__nv_bfloat16)));
  CKM(cudaMemcpy(mlp->prm, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice));
  CKM(cudaMemset(mlp->grad, 0, mlp::NPARAM * sizeof(float)));
  CKM(cudaMemset(mlp->m1, 0, mlp::NPARAM * sizeof(float)));
  CKM(cudaMemset(mlp->m2, 0, mlp::NPARAM * sizeof(float)));
  for (int i = 0; i < mlp::IN; ++i) mlp->norm[mlp::IN + i] = 1.0f;
  for (int i = 0; i < mlp::OUT; ++i) mlp->norm[2 * mlp::IN + mlp::OUT + i] = 1.0f;
  int r = mlp_refresh_bf16(mlp);
  if (r) return r;
  CKM(cudaDeviceSynchronize());
  *out = mlp;
  return IMEX_OK;
}

int imex_mlp_destroy(ImexMLP* mlp) {
  if (!mlp) return IMEX_EINVAL;
  cudaSetDevice(mlp->device);
  void* b[] = {mlp->prm, mlp->grad, mlp->m1, mlp->m2, mlp->loss, mlp->bw};
  for (void* x : b)
    if (x) cudaFree(x);
  delete mlp;
  return IMEX_OK;
}

int imex_mlp_get_params(ImexMLP* mlp, float* params) {
  if (!mlp || !params) return IMEX_EINVAL;
  CKM(cudaSetDevice(mlp->device));
  CKM(cudaMemcpy(params, mlp->prm, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  return IMEX_OK;
}

int imex_mlp_set_params(ImexMLP* mlp, const float* params) {
  if (!mlp || !params) return IMEX_EINVAL;
  CKM(cudaSetDevice(mlp->device));
  CKM(cudaMemcpy(mlp->prm, params, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  int r = mlp_refresh_bf16(mlp);
  if (r) return r;
  CKM(cudaDeviceSynchronize());
  return IMEX_OK;
}

int imex_mlp_set_norm(ImexMLP* mlp, const float* norm) {
  if (!mlp || !norm) return IMEX_EINVAL;
  for (int i = 0; i < 2 * mlp::IN + 2 * mlp::OUT; ++i) mlp->norm[i] = norm[i];
  return IMEX_OK;
}

int imex_mlp_get_norm(ImexMLP* mlp, float* norm) {
  if (!mlp || !norm) return IMEX_EINVAL;
  for (int i = 0; i < 2 * mlp::IN + 2 * mlp::OUT; ++i) norm[i] = mlp->norm[i];
  return IMEX_OK;
}

int imex_mlp_predict(ImexMLP* mlp, const float* x, int64_t n, float* y) {
  if (!mlp || !x || !y || n < 0) return IMEX_EINVAL;
  if (n == 0) return IMEX_OK;
  CKM(cudaSetDevice(mlp->device));
  float *dx = nullptr, *dy = nullptr;
  CKM(cudaMalloc((void**)&dx, n * mlp::IN * sizeof(float)));
  CKM(cudaMalloc((void**)&dy, n * mlp::OUT * sizeof(float)));
  CKM(cudaMemcpy(dx, x, n * mlp::IN * sizeof(float), cudaMemcpyHostToDevice));
  CKM(cudaFuncSetAttribute(mlp::k_mlp_predict, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)mlp::SMEM_NET));
  const long long tiles = (n + mlp::SAMPLES - 1) / mlp::SAMPLES;
  mlp::k_mlp_predict<<<(int)std::min<long long>(tiles, 148 * 4), 32 * mlp::WARPS, mlp::SMEM_NET>>>(
      mlp->bw, mlp->prm, dx, dy, n);
  CKM(cudaGetLastError());
  CKM(cudaMemcpy(y, dy, n * mlp::OUT * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(dx);
  cudaFree(dy);
  return IMEX_OK;
}

int imex_mlp_loss_grad(ImexMLP* mlp, const float* x, const float* y, int64_t n, float* loss,
                       float* grad) {
  if (!mlp || !x || !y || n <= 0) return IMEX_EINVAL;
  CKM(cudaSetDevice(mlp->device));
  float *dx = nullptr, *dy = nullptr;
  CKM(cudaMalloc((void**)&dx, n * mlp::IN * sizeof(float)));
  CKM(cudaMalloc((void**)&dy, n * mlp::OUT * sizeof(float)));
  CKM(cudaMemcpy(dx, x, n * mlp::IN * sizeof(float), cudaMemcpyHostToDevice));
  CKM(cudaMemcpy(dy, y, n * mlp::OUT * sizeof(float), cudaMemcpyHostToDevice));
  CKM(cudaMemset(mlp->grad, 0, mlp::NPARAM * sizeof(float)));
  int r = mlp_grad_pass(mlp, dx, dy, n);
  if (r) return r;
  float ls = 0.0f;
  CKM(cudaMemcpy(&ls, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) *loss = ls / (float)(n * mlp::OUT);
  if (grad) CKM(cudaMemcpy(grad, mlp->grad, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
  CKM(cudaMemset(mlp->grad, 0, mlp::NPARAM * sizeof(float)));
  cudaFree(dx);
  cudaFree(dy);
  return IMEX_OK;
}

// Adam on mini-batches of a device-resident training set (normalised x, y),
// shuffled once with `seed`; loss_out[e] = mean squared error of epoch e.
int imex_mlp_train(ImexMLP* mlp, const float* x_dev, const float* y_dev, int64_t n, int epochs,
                   int batch, float lr, uint64_t seed, float* loss_out) {
  if (!mlp || !x_dev || !y_dev || n <= 0 || epochs < 0 || batch <= 0) return IMEX_EINVAL;
  CKM(cudaSetDevice(mlp->device));
  std::vector<long long> perm(n);
  for (long long i = 0; i < n; ++i) perm[i] = i;
  uint64_t st = seed;
  for (long long i = n - 1; i > 0; --i) {
    long long j = (long long)(splitmix64(st) % (uint64_t)(i + 1));
    std::swap(perm[i], perm[j]);
  }
  long long* dperm = nullptr;
  float *xs = nullptr, *ys = nullptr;
  CKM(cudaMalloc((void**)&dperm, n * sizeof(long long)));
  CKM(cudaMalloc((void**)&xs, n * mlp::IN * sizeof(float)));
  CKM(cudaMalloc((void**)&ys, n * mlp::OUT * sizeof(float)));
  CKM(cudaMemcpy(dperm, perm.data(), n * sizeof(long long), cudaMemcpyHostToDevice));
  mlp::k_gather_rows<<<148 * 8, 256>>>(x_dev, dperm, xs, n, mlp::IN);
  mlp::k_gather_rows<<<148 * 8, 256>>>(y_dev, dperm, ys, n, mlp::OUT);
  CKM(cudaGetLastError());
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int e = 0; e < epochs; ++e) {
    double esum = 0.0;
    for (long long b0 = 0; b0 < n; b0 += batch) {
      const long long nb = std::min<long long>(batch, n - b0);
      int r = mlp_grad_pass(mlp, xs + b0 * mlp::IN, ys + b0 * mlp::OUT, nb);
      if (r) return r;
      ++mlp->adam_t;
      const float c1 = 1.0f - std::pow(b1, (float)mlp->adam_t);
      const float c2 = 1.0f - std::pow(b2, (float)mlp->adam_t);
      mlp::k_mlp_adam<<<(mlp::NPARAM + 255) / 256, 256>>>(mlp->prm, mlp->grad, mlp->m1, mlp->m2,
                                                           lr, b1, b2, eps, c1, c2);
      r = mlp_refresh_bf16(mlp);
      if (r) return r;
      float ls = 0.0f;
      CKM(cudaMemcpy(&ls, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost));
      esum += ls;
    }
    if (loss_out) loss_out[e] = (float)(esum / (double)(n * mlp::OUT));
  }
  CKM(cudaDeviceSynchronize());
  cudaFree(dperm);
  cudaFree(xs);
  cudaFree(ys);
  return IMEX_OK;
}

const char* imex_mlp_last_error(ImexMLP* mlp) { return mlp ? mlp->last_error.c_str() : "null"; }

}  // extern "C"

// ============================================================ warm start
namespace {
template <int NS>
cudaError_t launch_warm_predict_ns(ImexCtx* ctx) {
  static std::atomic<unsigned long long> attr{0};
  if (attr_needed(attr)) {
    cudaError_t e = cudaFuncSetAttribute(k_warm_predict<NS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mlp::SMEM_NET);
    if (e != cudaSuccess) return e;
    attr_done(attr);
  }
  WarmNorm nrm;
  const float* n = ctx->warm_mlp->norm;
  for (int i = 0; i < WARM_IN; ++i) {
    nrm.x_mean[i] = n[i];
    nrm.x_std[i] = n[WARM_IN + i];
  }
  for (int i = 0; i < WARM_OUT; ++i) {
    nrm.y_mean[i] = n[2 * WARM_IN + i];
    nrm.y_std[i] = n[2 * WARM_IN + WARM_OUT + i];
  }
  k_warm_predict<NS><<<148 * 2, 32 * mlp::WARPS, mlp::SMEM_NET, ctx->stream>>>(
      ctx->P, ctx->nw, ctx->clk, ctx->warm_mlp->bw, ctx->warm_mlp->prm, nrm);
  ctx->launches += 1;
  return cudaGetLastError();
}

cudaError_t launch_warm_predict(ImexCtx* ctx) {
  switch (ctx->ns) {
    case 1: return launch_warm_predict_ns<1>(ctx);
    case 2: return launch_warm_predict_ns<2>(ctx);
    case 3: return launch_warm_predict_ns<3>(ctx);
    default: return launch_warm_predict_ns<4>(ctx);
  }
}
}  // namespace

static void drop_graph(ImexCtx* ctx) {
  if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
  if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
}

extern "C" {

int imex_gpu_set_warmstart(ImexCtx* ctx, ImexMLP* net) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  if (net && net->device != ctx->device)
    return fail(ctx, IMEX_EINVAL, "imex_gpu_set_warmstart: network on another device");
  const size_t plane = (size_t)ctx->P.plane;
  if (net && !ctx->nw_wlist) {
    CK(dalloc(&ctx->nw_wlist, plane * 2));   // warm-start list, then fallback list
    CK(dalloc(&ctx->nw_feat, plane * WARM_IN));
    CK(dalloc(&ctx->nw_guess, plane * 2));
  }
  ctx->warm_mlp = net;
  ctx->nw.warm = net ? 1 : 0;
  ctx->nw.wlist = ctx->nw_wlist;
  ctx->nw.flist = ctx->nw_wlist ? ctx->nw_wlist + plane : nullptr;
  ctx->nw.feat = ctx->nw_feat;
  ctx->nw.guess = ctx->nw_guess;
  drop_graph(ctx);
  return IMEX_OK;
}

int imex_gpu_harvest_start(ImexCtx* ctx, int64_t capacity, int stride) {
  if (!ctx || capacity <= 0 || stride < 1) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->h_x) cudaFree(ctx->h_x);
  if (ctx->h_y) cudaFree(ctx->h_y);
  ctx->h_x = nullptr;
  ctx->h_y = nullptr;
  CK(dalloc(&ctx->h_x, (size_t)capacity * WARM_IN));
  CK(dalloc(&ctx->h_y, (size_t)capacity * WARM_OUT));
  ctx->nw.harvest = 1;
  ctx->nw.hstride = (unsigned int)stride;
  ctx->nw.hcap = (unsigned long long)capacity;
  ctx->nw.hx = ctx->h_x;
  ctx->nw.hy = ctx->h_y;
  const unsigned long long zero = 0;
  CK(cudaMemcpy(&ctx->clk->harvest_n, &zero, sizeof(zero), cudaMemcpyHostToDevice));
  drop_graph(ctx);
  return IMEX_OK;
}

int imex_gpu_harvest_stop(ImexCtx* ctx) {
  if (!ctx) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->nw.harvest = 0;
  drop_graph(ctx);
  return IMEX_OK;
}

int imex_gpu_harvest_data(ImexCtx* ctx, const float** x_dev, const float** y_dev, int64_t* n) {
  if (!ctx || !n) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  unsigned long long cnt = 0;
  CK(cudaMemcpy(&cnt, &ctx->clk->harvest_n, sizeof(cnt), cudaMemcpyDeviceToHost));
  *n = (int64_t)std::min<unsigned long long>(cnt, ctx->nw.hcap);
  if (x_dev) *x_dev = ctx->h_x;
  if (y_dev) *y_dev = ctx->h_y;
  return IMEX_OK;
}

}  // extern "C"

// ================================================================ ensemble
// Many independent runs (members) on one GPU, each with its own grid and
// parameters: one context per member, all members' time steps captured into
// one CUDA graph and replayed.  The graph forks the members over K streams
// (members dealt largest first to the least loaded stream); K is chosen by
// timing the first steps with K = 1, 2, 4, ... (each a real step: members
// are independent, so the results do not depend on K).
struct ImexEnsemble {
  int device = 0;
  std::vector<ImexCtx*> members;
  cudaStream_t root = nullptr;
  std::vector<cudaStream_t> workers;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<int64_t> step_launches;  // per member: kernels in one replayed step
  int k_streams = 0;                 // chosen concurrency (0: not tuned yet)
  std::vector<int> tried_k;
  std::vector<float> tried_ms;
  std::string last_error;
  // batched mode: every phase one persistent kernel for all members
  // (imex_batch.cuh); the tile shape is chosen by timing a real step with each
  int shape = -1;                    // chosen index into kShapes (-1: not tuned yet)
  int batch_shape = -1;              // shape the device tables are built for
  std::vector<int> tried_shape;
  std::vector<float> tried_shape_ms;
  void* dM = nullptr;                // device member table (imex_batch_api.h)
  uint32_t* tile_member = nullptr;
  uint32_t* active = nullptr;
  unsigned int* n_active = nullptr;
  unsigned long long* list_off = nullptr;
  long long n_tiles = 0;
  size_t tile_cap = 0;               // capacity of tile_member / active
  int64_t batch_launches = 0;        // kernels in one batched step
  int graph_shape = -1;              // tile shape of the captured graph (-1: per-member graph)
  int mode = 0;                      // 0 batched when possible, 2 per-member graphs
};

namespace {

constexpr int ENS_MAX_STREAMS = 32;

int ens_fail(ImexEnsemble* e, int code, const std::string& msg) {
  if (e) e->last_error = msg;
  return code;
}

#define CKE(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) return ens_fail(ens, IMEX_ECUDA, cudaGetErrorString(e_)); \
  } while (0)

void ens_drop_graph(ImexEnsemble* ens);

// Tile shapes the tuner tries for the batched mode.
struct ShapeDesc {
  int tx, ty;
};
constexpr ShapeDesc kShapes[3] = {{32, 8}, {16, 16}, {32, 4}};

// Batched mode needs one solid-class count for all members and none of the
// per-context extras (learned start, harvest, output sweep, moving bed).
bool ens_batchable(const ImexEnsemble* ens) {
  const int ns = ens->members[0]->ns;
  for (const ImexCtx* c : ens->members)
    if (c->ns != ns || c->nw.warm || c->nw.harvest || c->post_on || c->P.topo_change_flag)
      return false;
  return true;
}

// Member table and tile table for tile shape `si`.
int ens_build_tables(ImexEnsemble* ens, int si) {
  const int n = (int)ens->members.size();
  const int tx = kShapes[si].tx, ty = kShapes[si].ty;
  const size_t mb = imex_batch::member_bytes();
  std::vector<unsigned char> hM(mb * n);
  std::vector<uint32_t> tm;
  long long tile0 = 0;
  for (int m = 0; m < n; ++m) {
    ImexCtx* c = ens->members[m];
    imex_batch::MemberSrc d{};
    d.params = &c->P;
    d.params_bytes = sizeof(DevParams);
    d.newton_work = &c->nw;
    d.newton_work_bytes = sizeof(NewtonWork);
    d.q = c->q;
    d.X = c->X;
    d.mask = c->mask;
    d.cellinfo = c->cellinfo;
    d.release = c->release;
    d.Bx = c->Bx; d.By = c->By; d.Bxx = c->Bxx; d.Bxy = c->Bxy; d.Byy = c->Byy;
    d.gc = c->gc; d.dgc = c->dgc; d.gcsx = c->gcsx; d.gcsy = c->gcsy;
    d.ring = c->ring;
    d.erodible = c->erodible; d.deposit = c->deposit; d.erosion = c->erosion; d.Bcent = c->Bcent;
    d.clk = c->clk;
    d.exchange = erosion_active(c) ? 1 : 0;
    d.tiles_x = (c->P.nx + tx - 1) / tx;
    const long long tiles = (long long)d.tiles_x * ((c->P.ny + ty - 1) / ty);
    d.tile0 = tile0;
    if (!imex_batch::fill_member(hM.data() + mb * m, d))
      return ens_fail(ens, IMEX_EINVAL, "member record layout differs between units");
    tm.insert(tm.end(), (size_t)tiles, (uint32_t)m);
    tile0 += tiles;
  }
  if (tile0 > (long long)UINT32_MAX) return ens_fail(ens, IMEX_EUNSUPPORTED, "too many tiles");
  if (!ens->dM) CKE(cudaMalloc(&ens->dM, mb * n));
  if (!ens->list_off) CKE(cudaMalloc((void**)&ens->list_off, sizeof(unsigned long long) * (n + 1)));
  if (!ens->n_active) CKE(cudaMalloc((void**)&ens->n_active, sizeof(unsigned int)));
  if ((size_t)tile0 > ens->tile_cap) {
    if (ens->tile_member) cudaFree(ens->tile_member);
    if (ens->active) cudaFree(ens->active);
    ens->tile_member = nullptr;
    ens->active = nullptr;
    CKE(cudaMalloc((void**)&ens->tile_member, sizeof(uint32_t) * tile0));
    CKE(cudaMalloc((void**)&ens->active, sizeof(uint32_t) * tile0));
    ens->tile_cap = (size_t)tile0;
  }
  CKE(cudaMemcpy(ens->dM, hM.data(), mb * n, cudaMemcpyHostToDevice));
  CKE(cudaMemcpy(ens->tile_member, tm.data(), sizeof(uint32_t) * tile0, cudaMemcpyHostToDevice));
  ens->n_tiles = tile0;
  ens->batch_shape = si;
  return IMEX_OK;
}

int sm_count(int device) {
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n > 0 ? n : 148;
}

// One batched step of every member on ens->root (imex_batch.cu).
cudaError_t ens_enqueue_batch(ImexEnsemble* ens, int si) {
  imex_batch::Launch L{};
  L.members = ens->dM;
  L.n_members = (int)ens->members.size();
  L.ns = ens->members[0]->ns;
  L.shape = si;
  L.tile_member = ens->tile_member;
  L.active = ens->active;
  L.n_active = ens->n_active;
  L.list_off = ens->list_off;
  L.n_tiles = ens->n_tiles;
  L.any_exchange = 0;
  for (const ImexCtx* c : ens->members)
    if (erosion_active(c)) L.any_exchange = 1;
  L.sms = sm_count(ens->device);
  L.stream = ens->root;
  int launches = 0;
  cudaError_t e = imex_batch::enqueue_step(L, &launches);
  ens->batch_launches = launches;
  return e;
}

// Capture one batched step (tile shape si) into ens->graph.
int ens_build_batch_graph(ImexEnsemble* ens, int si) {
  ens_drop_graph(ens);
  if (ens->batch_shape != si) {
    int r = ens_build_tables(ens, si);
    if (r) return r;
  }
  CKE(cudaStreamBeginCapture(ens->root, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = ens_enqueue_batch(ens, si);
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(ens->root, &g);
  if (err != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ens_fail(ens, IMEX_ECUDA, cudaGetErrorString(err));
  }
  if (e2 != cudaSuccess) return ens_fail(ens, IMEX_ECUDA, cudaGetErrorString(e2));
  ens->graph = g;
  CKE(cudaGraphInstantiate(&ens->exec, g, 0));
  ens->step_launches.assign(ens->members.size(), ens->batch_launches);
  ens->graph_shape = si;
  return IMEX_OK;
}

void ens_drop_graph(ImexEnsemble* ens) {
  if (ens->exec) cudaGraphExecDestroy(ens->exec);
  if (ens->graph) cudaGraphDestroy(ens->graph);
  ens->exec = nullptr;
  ens->graph = nullptr;
}

// Capture one step of every member, forked over k streams.
int ens_build_graph(ImexEnsemble* ens, int k) {
  ens_drop_graph(ens);
  const int n = (int)ens->members.size();
  std::vector<int> order(n);
  for (int m = 0; m < n; ++m) order[m] = m;
  auto cells = [&](int m) { return (double)ens->members[m]->P.nx * ens->members[m]->P.ny; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells(a) > cells(b); });
  std::vector<std::vector<int>> bucket(k);
  std::vector<double> load(k, 0.0);
  for (int m : order) {
    int best = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    bucket[best].push_back(m);
    load[best] += cells(m);
  }
  std::vector<int64_t> l0(n);
  for (int m = 0; m < n; ++m) l0[m] = ens->members[m]->launches;
  CKE(cudaStreamBeginCapture(ens->root, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaEventRecord(ens->fork, ens->root);
  for (int w = 0; w < k && err == cudaSuccess; ++w) {
    err = cudaStreamWaitEvent(ens->workers[w], ens->fork, 0);
    for (int m : bucket[w]) {
      if (err != cudaSuccess) break;
      ImexCtx* c = ens->members[m];
      cudaStream_t saved = c->stream;
      c->stream = ens->workers[w];
      err = enqueue_step(c);
      c->stream = saved;
    }
    if (err == cudaSuccess) err = cudaEventRecord(ens->join[w], ens->workers[w]);
    if (err == cudaSuccess) err = cudaStreamWaitEvent(ens->root, ens->join[w], 0);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(ens->root, &g);
  if (err != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ens_fail(ens, IMEX_ECUDA, cudaGetErrorString(err));
  }
  if (e2 != cudaSuccess) return ens_fail(ens, IMEX_ECUDA, cudaGetErrorString(e2));
  ens->graph = g;
  CKE(cudaGraphInstantiate(&ens->exec, g, 0));
  ens->graph_shape = -1;
  // the capture counted each member's kernels once; replays count them
  ens->step_launches.assign(n, 0);
  for (int m = 0; m < n; ++m) {
    ens->step_launches[m] = ens->members[m]->launches - l0[m];
    ens->members[m]->launches = l0[m];
  }
  return IMEX_OK;
}

int ens_replay(ImexEnsemble* ens, float* ms) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (ms) {
    CKE(cudaEventCreate(&a));
    CKE(cudaEventCreate(&b));
    CKE(cudaEventRecord(a, ens->root));
  }
  CKE(cudaGraphLaunch(ens->exec, ens->root));
  for (size_t m = 0; m < ens->members.size(); ++m) ens->members[m]->launches += ens->step_launches[m];
  if (ms) {
    CKE(cudaEventRecord(b, ens->root));
    CKE(cudaEventSynchronize(b));
    CKE(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  return IMEX_OK;
}

}  // namespace

extern "C" {

int imex_gpu_ensemble_create(int n_members, const ImexParams* const* params,
                             const ImexStatic* const* statics, int device, ImexEnsemble** out) {
  if (!out || n_members < 1 || !params || !statics) return IMEX_EINVAL;
  *out = nullptr;
  ImexEnsemble* ens = new ImexEnsemble();
  for (int m = 0; m < n_members; ++m) {
    ImexCtx* c = nullptr;
    int r = imex_gpu_create(params[m], statics[m], device, &c);
    if (r != IMEX_OK) {
      for (ImexCtx* x : ens->members) imex_gpu_destroy(x);
      delete ens;
      return r;
    }
    ens->members.push_back(c);
  }
  ens->device = ens->members[0]->device;
  CKE(cudaSetDevice(ens->device));
  CKE(cudaStreamCreateWithFlags(&ens->root, cudaStreamNonBlocking));
  const int nw = std::min(n_members, ENS_MAX_STREAMS);
  ens->workers.resize(nw);
  ens->join.resize(nw);
  for (int w = 0; w < nw; ++w) {
    CKE(cudaStreamCreateWithFlags(&ens->workers[w], cudaStreamNonBlocking));
    CKE(cudaEventCreateWithFlags(&ens->join[w], cudaEventDisableTiming));
  }
  CKE(cudaEventCreateWithFlags(&ens->fork, cudaEventDisableTiming));
  *out = ens;
  return IMEX_OK;
}

int imex_gpu_ensemble_destroy(ImexEnsemble* ens) {
  if (!ens) return IMEX_EINVAL;
  cudaSetDevice(ens->device);
  if (ens->root) cudaStreamSynchronize(ens->root);
  ens_drop_graph(ens);
  for (cudaStream_t w : ens->workers) cudaStreamDestroy(w);
  for (cudaEvent_t e : ens->join) cudaEventDestroy(e);
  if (ens->fork) cudaEventDestroy(ens->fork);
  if (ens->root) cudaStreamDestroy(ens->root);
  if (ens->dM) cudaFree(ens->dM);
  if (ens->tile_member) cudaFree(ens->tile_member);
  if (ens->active) cudaFree(ens->active);
  if (ens->n_active) cudaFree(ens->n_active);
  if (ens->list_off) cudaFree(ens->list_off);
  for (ImexCtx* c : ens->members) imex_gpu_destroy(c);
  delete ens;
  return IMEX_OK;
}

int imex_gpu_ensemble_member(ImexEnsemble* ens, int m, ImexCtx** ctx) {
  if (!ens || !ctx || m < 0 || m >= (int)ens->members.size()) return IMEX_EINVAL;
  *ctx = ens->members[m];
  return IMEX_OK;
}

int imex_gpu_ensemble_advance(ImexEnsemble* ens, int n_steps, int* first_bad_member) {
  if (!ens || n_steps < 0) return IMEX_EINVAL;
  CKE(cudaSetDevice(ens->device));
  if (first_bad_member) *first_bad_member = -1;
  // members' own work (set_state, set_clock) is ordered before the graph
  for (ImexCtx* c : ens->members) CKE(cudaStreamSynchronize(c->stream));
  const int nmem = (int)ens->members.size();
  int done = 0;
  const bool batched = ens->mode != 2 && ens_batchable(ens);
  if (batched) {
    // batched mode; tuning: real steps with the tile shapes in the order
    // 0 1 2 2 1 0, so that a step cost that drifts linearly as the currents
    // spread weighs on every shape alike; the smallest sum wins
    constexpr int n_shapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
    while (ens->shape < 0 && done < n_steps) {
      const int k = (int)ens->tried_shape.size();
      const int si = k < n_shapes ? k : 2 * n_shapes - 1 - k;
      int r = ens_build_batch_graph(ens, si);
      if (r) return r;
      float ms = 0.0f;
      r = ens_replay(ens, &ms);
      if (r) return r;
      ens->tried_shape.push_back(si);
      ens->tried_shape_ms.push_back(ms);
      ++done;
      if ((int)ens->tried_shape.size() == 2 * n_shapes) {
        double sum[n_shapes] = {0.0};
        for (size_t i = 0; i < ens->tried_shape.size(); ++i)
          sum[ens->tried_shape[i]] += ens->tried_shape_ms[i];
        int best = 0;
        for (int i = 1; i < n_shapes; ++i)
          if (sum[i] < sum[best]) best = i;
        ens->shape = best;
      }
    }
    if (done < n_steps && ens->shape < 0) ens->shape = ens->tried_shape.back();
    if (done < n_steps) {
      if (!ens->exec || ens->batch_shape != ens->shape || ens->graph_shape != ens->shape) {
        int r = ens_build_batch_graph(ens, ens->shape);
        if (r) return r;
      }
      for (; done < n_steps; ++done) {
        int r = ens_replay(ens, nullptr);
        if (r) return r;
      }
    }
  }
  // tuning: one real step per candidate stream count
  while (!batched && ens->k_streams == 0 && done < n_steps) {
    int k = ens->tried_k.empty() ? 1 : ens->tried_k.back() * 2;
    if (k > std::min(nmem, ENS_MAX_STREAMS)) {
      size_t best = 0;
      for (size_t i = 1; i < ens->tried_ms.size(); ++i)
        if (ens->tried_ms[i] < ens->tried_ms[best]) best = i;
      ens->k_streams = ens->tried_k[best];
      break;
    }
    int r = ens_build_graph(ens, k);
    if (r) return r;
    float ms = 0.0f;
    r = ens_replay(ens, &ms);
    if (r) return r;
    ens->tried_k.push_back(k);
    ens->tried_ms.push_back(ms);
    ++done;
  }
  if (done < n_steps) {
    if (!ens->exec || ens->graph_shape >= 0 || ens->tried_k.empty() ||
        ens->tried_k.back() != ens->k_streams) {
      int r = ens_build_graph(ens, ens->k_streams);
      if (r) return r;
      ens->tried_k.push_back(ens->k_streams);
      ens->tried_ms.push_back(-1.0f);
    }
    for (; done < n_steps; ++done) {
      int r = ens_replay(ens, nullptr);
      if (r) return r;
    }
  }
  CKE(cudaStreamSynchronize(ens->root));
  int first = IMEX_OK;
  for (int m = 0; m < nmem; ++m) {
    ImexCtx* c = ens->members[m];
    c->x_valid = false;
    int r = collect_errors(c);
    if (r != IMEX_OK && first == IMEX_OK) {
      first = r;
      if (first_bad_member) *first_bad_member = m;
    }
  }
  return first;
}

int imex_gpu_ensemble_tuning(ImexEnsemble* ens, int* k_streams, int* n_tried, int* tried_k,
                             float* tried_ms, int cap) {
  if (!ens) return IMEX_EINVAL;
  if (k_streams) *k_streams = ens->k_streams;
  int n = 0;
  for (size_t i = 0; i < ens->tried_k.size(); ++i) {
    if (ens->tried_ms[i] < 0.0f) continue;
    if (n < cap) {
      if (tried_k) tried_k[n] = ens->tried_k[i];
      if (tried_ms) tried_ms[n] = ens->tried_ms[i];
    }
    ++n;
  }
  if (n_tried) *n_tried = n;
  return IMEX_OK;
}

int imex_gpu_ensemble_set_mode(ImexEnsemble* ens, int mode) {
  if (!ens || (mode != 0 && mode != 2)) return IMEX_EINVAL;
  if (mode == ens->mode) return IMEX_OK;
  CKE(cudaSetDevice(ens->device));
  CKE(cudaStreamSynchronize(ens->root));
  ens_drop_graph(ens);
  ens->mode = mode;
  return IMEX_OK;
}

int imex_gpu_ensemble_tile_shape(ImexEnsemble* ens, int* tx, int* ty, int* n_tried,
                                 int* tried_tx, int* tried_ty, float* tried_ms, int cap) {
  if (!ens) return IMEX_EINVAL;
  if (tx) *tx = ens->shape >= 0 ? kShapes[ens->shape].tx : 0;
  if (ty) *ty = ens->shape >= 0 ? kShapes[ens->shape].ty : 0;
  const int n = (int)ens->tried_shape.size();
  for (int i = 0; i < n && i < cap; ++i) {
    if (tried_tx) tried_tx[i] = kShapes[ens->tried_shape[i]].tx;
    if (tried_ty) tried_ty[i] = kShapes[ens->tried_shape[i]].ty;
    if (tried_ms) tried_ms[i] = ens->tried_shape_ms[i];
  }
  if (n_tried) *n_tried = n;
  return IMEX_OK;
}

const char* imex_gpu_ensemble_last_error(ImexEnsemble* ens) {
  return ens ? ens->last_error.c_str() : "null ensemble";
}

}  // extern "C"

// ======================================================= allocation-free dt
// imex_gpu_timestep_noalloc: the CFL time step of imex_gpu_timestep for
// callers that may not allocate device memory when they call it, e.g. a
// driver whose GPU memory is a fixed pool owned by another framework, where
// a new allocation would fail or break the pool's accounting.  It allocates
// nothing: its only scratch is the file-scope array below, one partial
// minimum per 32x8 tile plus one result slot.  Every call writes all the
// slots it later reads, so nothing needs to start at zero; calls that run at
// the same time on one GPU share the array and race.
namespace {
constexpr int NOALLOC_MAX_TILES = 1 << 20;  // 8 MiB of doubles + 1 result slot
}  // namespace
static __device__ __align__(256) double g_noalloc_dt[NOALLOC_MAX_TILES + 1];

namespace {
// Device address of g_noalloc_dt, looked up once per device (host code may
// not use the symbol's name as a device address).
// Atomic, so that two host threads making their first call on one device
// at once both store the same address without a data race.
constexpr int NOALLOC_MAX_DEVICES = 64;
std::atomic<double*> g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Per-tile CFL minimum.  k_flux takes its speeds from the stage view and,
// when an inlet-interior cell is in the stencil, from the timestep view;
// the two views differ only at inlet-interior cells, so taking the timestep
// view everywhere gives the same speeds.  The fluxes are discarded.
template <int NS>
__global__ void __launch_bounds__(FLUX_THREADS)
    k_cfl_tiles(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                const uint8_t* __restrict__ mask, const uint8_t* __restrict__ cellinfo,
                const double* __restrict__ gcsx, const double* __restrict__ gcsy,
                const RingCell* __restrict__ ring, const DevClock* clk, double* tile_min) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const DevParams& P = Pp;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  CflShared<NS>& S = *reinterpret_cast<CflShared<NS>*>(smem_raw);
  const int j0 = blockIdx.x * TX, k0 = blockIdx.y * TY;
  const int nx = P.nx, ny = P.ny;
  const long long tile = (long long)blockIdx.y * gridDim.x + blockIdx.x;
  const double time = clk->t;
  int any = 0;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    int j = j0 + e % TX, k = k0 + e / TX;
    if (j < nx && k < ny && mask[(size_t)k * P.pitch + j]) any = 1;
  }
  if (!__syncthreads_or(any)) {
    if (threadIdx.x == 0) tile_min[tile] = P.max_dt;
    return;
  }
  for (int e = threadIdx.x; e < SW * SH; e += blockDim.x) {
    int lx = e % SW, ly = e / SW;
    int j = j0 + lx - HALO, k = k0 + ly - HALO;
    double qc[NV], qpv[NP];
    uint8_t inf = 0;
    if (j >= 0 && j < nx && k >= 0 && k < ny) {
      size_t c = (size_t)k * P.pitch + j;
      inf = P.has_cellinfo ? cellinfo[(size_t)k * nx + j] : 0;
      if (mask[c]) inf |= 128;
      if (P.radial_source_flag && (inf & CI_SRC_MASK) == 1) {
#pragma unroll
        for (int i = 0; i < NP; ++i) qpv[i] = 0.0;
        qpv[3] = P.T_ambient;
      } else {
#pragma unroll
        for (int i = 0; i < NV; ++i) qc[i] = q[c + (size_t)i * P.plane];
        cell_qp<NS>(P, qc, qpv);
      }
    } else {
#pragma unroll
      for (int i = 0; i < NP; ++i) qpv[i] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < NP; ++i) S.tile.qp[i][ly][lx] = qpv[i];
    S.tile.info[ly][lx] = inf;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < NXI + NYI; e += blockDim.x) {
    double H[NV], amax = 0.0, aN, aP;
    if (e < NXI) {
      int jj = e % (TX + 1), kk = e / (TX + 1);
      int ja = j0 + jj - 1, ka = k0 + kk, ia_x = jj - 1 + HALO, ia_y = kk + HALO;
      S.ax[kk][jj] = 0.0;
      if (ka >= ny || ja + 1 > nx || nx == 1) continue;
      bool a_in = ja >= 0, b_in = ja + 1 < nx;
      bool sa = a_in && (S.tile.info[ia_y][ia_x] & 128);
      bool sb = b_in && (S.tile.info[ia_y][ia_x + 1] & 128);
      if (!(sa || sb)) continue;
      double gcf = P.slope_correction_flag ? gcsx[(size_t)ka * (nx + 1) + (ja + 1)] : 1.0;
      interface_flux<NS>(P, S.tile, 1, ia_x, ia_y, ja, ka, a_in, b_in, gcf, false, time, ring, H,
                         amax, aN, aP);
      S.ax[kk][jj] = amax;
    } else {
      int e2 = e - NXI;
      int jj = e2 % TX, kk = e2 / TX;
      int ja = j0 + jj, ka = k0 + kk - 1, ia_x = jj + HALO, ia_y = kk - 1 + HALO;
      S.ay[kk][jj] = 0.0;
      if (ja >= nx || ka + 1 > ny || ny == 1) continue;
      bool a_in = ka >= 0, b_in = ka + 1 < ny;
      bool sa = a_in && (S.tile.info[ia_y][ia_x] & 128);
      bool sb = b_in && (S.tile.info[ia_y + 1][ia_x] & 128);
      if (!(sa || sb)) continue;
      double gcf = P.slope_correction_flag ? gcsy[(size_t)(ka + 1) * nx + ja] : 1.0;
      interface_flux<NS>(P, S.tile, 2, ia_x, ia_y, ja, ka, a_in, b_in, gcf, false, time, ring, H,
                         amax, aN, aP);
      S.ay[kk][jj] = amax;
    }
  }
  __syncthreads();
  double dtl = P.max_dt;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    int jj = e % TX, kk = e / TX;
    int j = j0 + jj, k = k0 + kk;
    if (j >= nx || k >= ny) continue;
    if (!(S.tile.info[kk + HALO][jj + HALO] & 128)) continue;
    double max_a = fmax_f(S.ax[kk][jj], S.ax[kk][jj + 1]);
    double dtx = (max_a > 0.0) ? P.cfl * P.dx / max_a : dtl;
    max_a = fmax_f(S.ay[kk][jj], S.ay[kk + 1][jj]);
    double dty = (max_a > 0.0) ? P.cfl * P.dy / max_a : dtl;
    dtl = fmin_f(dtl, fmin_f(dtx, dty));
  }
  for (int off = 16; off > 0; off >>= 1) dtl = fmin_f(dtl, __shfl_down_sync(0xffffffffu, dtl, off));
  if ((threadIdx.x & 31) == 0) S.dtmin[threadIdx.x >> 5] = dtl;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = S.dtmin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin_f(m, S.dtmin[w]);
    tile_min[tile] = m;
  }
}

// One block folds the tile minima into slot n_tiles of the same array with
// the rule of the atomic minimum in k_flux (only 0 <= m < max_dt lowers dt).
__global__ void __launch_bounds__(1024) k_cfl_fold(const __grid_constant__ DevParams Pp,
                                                   double* tile_min, long long n_tiles) {
  __shared__ double red[32];
  const double max_dt = Pp.max_dt;
  double m = max_dt;
  for (long long i = threadIdx.x; i < n_tiles; i += blockDim.x) {
    double v = tile_min[i];
    if (v >= 0.0 && v < max_dt) m = fmin_f(m, v);
  }
  for (int off = 16; off > 0; off >>= 1) m = fmin_f(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) r = fmin_f(r, red[w]);
    tile_min[n_tiles] = r;
  }
}

template <int NS>
cudaError_t launch_cfl_tiles(ImexCtx* ctx, double* scratch) {
  const DevParams& P = ctx->P;
  size_t smem = sizeof(CflShared<NS>);
  cudaError_t e = cudaFuncSetAttribute(k_cfl_tiles<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  k_cfl_tiles<NS><<<tile_grid(P), FLUX_THREADS, smem, ctx->stream>>>(
      ctx->P, ctx->q, ctx->mask, ctx->cellinfo, ctx->gcsx, ctx->gcsy, ctx->ring, ctx->clk,
      scratch);
  ctx->launches += 1;
  return cudaGetLastError();
}
}  // namespace

extern "C" int imex_gpu_timestep_noalloc(ImexCtx* ctx, double* dt) {
  if (!ctx || !dt) return IMEX_EINVAL;
  CK(cudaSetDevice(ctx->device));
  const dim3 g = tile_grid(ctx->P);
  const long long n_tiles = (long long)g.x * g.y;
  if (n_tiles > NOALLOC_MAX_TILES)
    return fail(ctx, IMEX_EINVAL,
                "imex_gpu_timestep_noalloc: grid needs " + std::to_string(n_tiles) +
                    " tiles of 32x8 cells; the built-in scratch holds at most " +
                    std::to_string(NOALLOC_MAX_TILES));
  if (ctx->device < 0 || ctx->device >= NOALLOC_MAX_DEVICES)
    return fail(ctx, IMEX_EINVAL, "imex_gpu_timestep_noalloc: device index out of range");
  double* scratch = g_noalloc_ptr[ctx->device].load(std::memory_order_acquire);
  if (!scratch) {
    // first call on this device: resolve the scratch array's device address
    void* ptr = nullptr;
    CK(cudaGetSymbolAddress(&ptr, g_noalloc_dt));
    scratch = static_cast<double*>(ptr);
    g_noalloc_ptr[ctx->device].store(scratch, std::memory_order_release);
  }
  if (ctx->P.cfl == -1.0) {
    *dt = ctx->P.max_dt;
    return IMEX_OK;
  }
  cudaError_t e;
  switch (ctx->ns) {
    case 1: e = launch_cfl_tiles<1>(ctx, scratch); break;
    case 2: e = launch_cfl_tiles<2>(ctx, scratch); break;
    case 3: e = launch_cfl_tiles<3>(ctx, scratch); break;
    default: e = launch_cfl_tiles<4>(ctx, scratch); break;
  }
  CK(e);
  k_cfl_fold<<<1, 1024, 0, ctx->stream>>>(ctx->P, scratch, n_tiles);
  ctx->launches += 1;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dt, scratch + n_tiles, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return IMEX_OK;
}

// ===================================================== set-up on the device
namespace {

thread_local std::string g_setup_error;

int setup_fail(int code, const std::string& msg) {
  g_setup_error = msg;
  return code;
}
#define CKS(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return setup_fail(IMEX_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Device buffers of one set-up call, freed on every return path.
struct SetupBufs {
  std::vector<void*> p;
  ~SetupBufs() {
    for (void* b : p) cudaFree(b);
  }
  template <class T>
  cudaError_t alloc(T** out, size_t n) {
    cudaError_t e = cudaMalloc((void**)out, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(*out);
    return e;
  }
};

// Grid spacing as init_grid: cell_size, or 1 along an axis of one cell
// (src/geometry_2d.f90:250-266).
SetupGrid setup_grid(int nx, int ny, double x0, double y0, double cell_size) {
  SetupGrid G;
  G.nx = nx;
  G.ny = ny;
  G.x0 = x0;
  G.y0 = y0;
  G.dx = nx > 1 ? cell_size : 1.0;
  G.dy = ny > 1 ? cell_size : 1.0;
  return G;
}

int grid_blocks(long long n, int threads) {
  return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 64));
}

struct EvTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EvTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace

extern "C" {

const char* imex_setup_last_error(void) { return g_setup_error.c_str(); }

int imex_setup_dem(int device, int ncols, int nrows, double xllcorner, double yllcorner,
                   double cellsize, double nodata, const double* z, int nx, int ny, double x0,
                   double y0, double cell_size, double* B_cent, int8_t* B_nodata,
                   float* kernel_ms) {
  g_setup_error.clear();
  if (!z || !B_cent || !B_nodata || ncols < 1 || nrows < 1 || nx < 1 || ny < 1)
    return setup_fail(IMEX_EINVAL, "imex_setup_dem: empty DEM or grid, or NULL array");
  if (ncols == 1 && nrows == 1)
    return setup_fail(IMEX_EINVAL, "imex_setup_dem: a DEM of one node cannot be interpolated");
  if (device >= 0) CKS(cudaSetDevice(device));
  // node coordinates: xllcorner + (j - 0.5)*cellsize (src/inpout_2d.f90:3579-3589)
  std::vector<double> x1(ncols), y1(nrows);
  for (int j = 1; j <= ncols; ++j) x1[j - 1] = xllcorner + ((double)j - 0.5) * cellsize;
  for (int k = 1; k <= nrows; ++k) y1[k - 1] = yllcorner + ((double)k - 0.5) * cellsize;
  const size_t nz = (size_t)ncols * nrows, nc = (size_t)nx * ny;
  SetupBufs B;
  double *dx1, *dy1, *dz, *dB;
  int8_t* dN;
  int* derr;
  CKS(B.alloc(&dx1, ncols));
  CKS(B.alloc(&dy1, nrows));
  CKS(B.alloc(&dz, nz));
  CKS(B.alloc(&dB, nc));
  CKS(B.alloc(&dN, nc));
  CKS(B.alloc(&derr, 1));
  CKS(cudaMemcpy(dx1, x1.data(), ncols * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemcpy(dy1, y1.data(), nrows * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemcpy(dz, z, nz * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemset(derr, 0, sizeof(int)));
  const SetupGrid G = setup_grid(nx, ny, x0, y0, cell_size);
  DemView D{ncols, nrows, dx1, dy1, dz, nodata};
  EvTimer t;
  CKS(cudaEventCreate(&t.a));
  CKS(cudaEventCreate(&t.b));
  CKS(cudaEventRecord(t.a));
  k_dem_to_grid<<<grid_blocks((long long)nc, 256), 256>>>(G, D, dB, dN, derr);
  CKS(cudaGetLastError());
  CKS(cudaEventRecord(t.b));
  CKS(cudaEventSynchronize(t.b));
  if (kernel_ms) CKS(cudaEventElapsedTime(kernel_ms, t.a, t.b));
  int err = 0;
  CKS(cudaMemcpy(&err, derr, sizeof(int), cudaMemcpyDeviceToHost));
  CKS(cudaMemcpy(B_cent, dB, nc * sizeof(double), cudaMemcpyDeviceToHost));
  CKS(cudaMemcpy(B_nodata, dN, nc, cudaMemcpyDeviceToHost));
  if (err & SETUP_ERR_NONFINITE)
    return setup_fail(IMEX_EINVAL, "imex_setup_dem: non-finite DEM or grid coordinates");
  if (err & SETUP_ERR_OUTSIDE)
    return setup_fail(IMEX_EINVAL,
                      "imex_setup_dem: cell centres west or south of the DEM's first node");
  return IMEX_OK;
}

int imex_setup_cell_fract(int device, int nx, int ny, double x0, double y0, double cell_size,
                          double xs, double ys, double rs, double r2s, double angle_deg,
                          double* cell_fract, float* kernel_ms) {
  g_setup_error.clear();
  if (!cell_fract || nx < 1 || ny < 1)
    return setup_fail(IMEX_EINVAL, "imex_setup_cell_fract: empty grid or NULL array");
  if (device >= 0) CKS(cudaSetDevice(device));
  const SetupGrid G = setup_grid(nx, ny, x0, y0, cell_size);
  // ang_rad = angles/180*ATAN(1)*4 with the host's libm (src/geometry_2d.f90:1696)
  const double ang_rad = ((angle_deg / 180.0) * std::atan(1.0)) * 4.0;
  const double ca = std::cos(ang_rad), sa = std::sin(ang_rad);
  const double R = (rs > r2s) ? rs : r2s;
  // cells whose box meets the bounding square (the test of :1727-1730)
  auto x_stag = [&](int J) { return G.x0 + (double)(J - 1) * G.dx; };
  auto y_stag = [&](int K) { return G.y0 + (double)(K - 1) * G.dy; };
  int jlo = -1, jhi = -2, klo = -1, khi = -2;
  for (int j = 1; j <= nx; ++j)
    if (!(x_stag(j + 1) < (xs - R)) && !(x_stag(j) > (xs + R))) {
      if (jlo < 0) jlo = j;
      jhi = j;
    }
  for (int k = 1; k <= ny; ++k)
    if (!(y_stag(k + 1) < (ys - R)) && !(y_stag(k) > (ys + R))) {
      if (klo < 0) klo = k;
      khi = k;
    }
  // subgrid offsets ((2h-1)/(2n) - 1/2)*dx (src/geometry_2d.f90:1711-1722)
  std::vector<double> xsub(CF_POINTS), ysub(CF_POINTS);
  for (int h = 1; h <= CF_POINTS; ++h) {
    const double u = (2.0 * (double)h - 1.0) / (2.0 * (double)CF_POINTS);
    xsub[h - 1] = (u - 0.5) * G.dx;
    ysub[h - 1] = (u - 0.5) * G.dy;
  }
  const size_t nc = (size_t)nx * ny;
  SetupBufs B;
  double *dxs, *dys, *dout;
  CKS(B.alloc(&dxs, CF_POINTS));
  CKS(B.alloc(&dys, CF_POINTS));
  CKS(B.alloc(&dout, nc));
  CKS(cudaMemcpy(dxs, xsub.data(), CF_POINTS * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemcpy(dys, ysub.data(), CF_POINTS * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemset(dout, 0, nc * sizeof(double)));
  EvTimer t;
  CKS(cudaEventCreate(&t.a));
  CKS(cudaEventCreate(&t.b));
  CKS(cudaEventRecord(t.a));
  if (jlo > 0 && klo > 0) {
    CellFractArgs A;
    A.G = G;
    A.j_lo = jlo - 1;
    A.k_lo = klo - 1;
    A.n_j = jhi - jlo + 1;
    A.n_k = khi - klo + 1;
    A.xs = xs;
    A.ys = ys;
    A.rs2 = rs * rs;
    A.r2s2 = r2s * r2s;
    A.cos_a = ca;
    A.sin_a = sa;
    const long long ncand = (long long)A.n_j * A.n_k;
    const int blocks = (int)std::min<long long>(ncand, 148LL * 16);
    k_cell_fract<<<blocks, CF_THREADS>>>(A, dxs, dys, dout);
    CKS(cudaGetLastError());
  }
  CKS(cudaEventRecord(t.b));
  CKS(cudaEventSynchronize(t.b));
  if (kernel_ms) CKS(cudaEventElapsedTime(kernel_ms, t.a, t.b));
  CKS(cudaMemcpy(cell_fract, dout, nc * sizeof(double), cudaMemcpyDeviceToHost));
  return IMEX_OK;
}

int imex_setup_regrid(int device, int ncols, int nrows, double xllcorner, double yllcorner,
                      double cellsize, double nodata, const double* fin, int nx, int ny,
                      double x0, double y0, double cell_size, double* fout, float* kernel_ms) {
  g_setup_error.clear();
  if (!fin || !fout || ncols < 1 || nrows < 1 || nx < 1 || ny < 1)
    return setup_fail(IMEX_EINVAL, "imex_setup_regrid: empty raster or grid, or NULL array");
  if (device >= 0) CKS(cudaSetDevice(device));
  // raster edges xllcorner + (j-1)*cellsize, j = 1..ncols+1 (src/inpout_2d.f90:5203-5213)
  std::vector<double> xin(ncols + 1), yin(nrows + 1);
  for (int j = 1; j <= ncols + 1; ++j) xin[j - 1] = xllcorner + (double)(j - 1) * cellsize;
  for (int k = 1; k <= nrows + 1; ++k) yin[k - 1] = yllcorner + (double)(k - 1) * cellsize;
  const size_t nr = (size_t)ncols * nrows, nc = (size_t)nx * ny;
  SetupBufs B;
  double *dxin, *dyin, *dfin, *dout;
  int* derr;
  CKS(B.alloc(&dxin, ncols + 1));
  CKS(B.alloc(&dyin, nrows + 1));
  CKS(B.alloc(&dfin, nr));
  CKS(B.alloc(&dout, nc));
  CKS(B.alloc(&derr, 1));
  CKS(cudaMemcpy(dxin, xin.data(), (ncols + 1) * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemcpy(dyin, yin.data(), (nrows + 1) * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemcpy(dfin, fin, nr * sizeof(double), cudaMemcpyHostToDevice));
  CKS(cudaMemset(derr, 0, sizeof(int)));
  RegridArgs A{nx, ny, x0, y0, cell_size, ncols, nrows, nodata};
  EvTimer t;
  CKS(cudaEventCreate(&t.a));
  CKS(cudaEventCreate(&t.b));
  CKS(cudaEventRecord(t.a));
  k_regrid<<<grid_blocks((long long)nc, 256), 256>>>(A, dxin, dyin, dfin, dout, derr);
  CKS(cudaGetLastError());
  CKS(cudaEventRecord(t.b));
  CKS(cudaEventSynchronize(t.b));
  if (kernel_ms) CKS(cudaEventElapsedTime(kernel_ms, t.a, t.b));
  int err = 0;
  CKS(cudaMemcpy(&err, derr, sizeof(int), cudaMemcpyDeviceToHost));
  CKS(cudaMemcpy(fout, dout, nc * sizeof(double), cudaMemcpyDeviceToHost));
  if (err) return setup_fail(IMEX_EINVAL, "imex_setup_regrid: non-finite raster or grid coordinates");
  return IMEX_OK;
}

}  // extern "C"

// ===================================================== output_solution writers
namespace {

// One output_solution call: which files, and where each staged plane sits in
// the pinned buffer (offsets in units of nx*ny doubles; -1 = not staged).
struct OutJob {
  std::string run;
  int idx = 0, nx = 0, ny = 0, ns = 0, nv = 0, threads = 1;
  double x0 = 0, y0 = 0, dx = 1, dy = 1, cell_size = 1, porosity = 0;
  bool cons = false, phys = false, esri = false, maxf = false, first = false;
  bool erosion = false, settling = false, topo = false;
  long q = -1, ers_c = -1, erd_c = -1, dep_c = -1, B_c = -1;   // .q_2d family
  long p2d = -1;                                               // .p_2d columns
  long esr = -1, dep_e = -1, ers_e = -1, hmax = -1;            // ESRI grids
  const double* buf = nullptr;
};

double out_x_comp(const OutJob& J, int j) {   // j 1-based (src/geometry_2d.f90:294-320)
  return 0.5 * ((J.x0 + (double)(j - 1) * J.dx) + (J.x0 + (double)j * J.dx));
}
double out_y_comp(const OutJob& J, int k) {
  return 0.5 * ((J.y0 + (double)(k - 1) * J.dy) + (J.y0 + (double)k * J.dy));
}

// Rows k = 1..ny of a column file, formatted by `threads` workers in bands
// and written in order; each line is x_comp, y_comp and `cols` values.
// kind 0: E20.12 ('(2e20.12,100(e20.12))'), kind 1: ES15.7E2 ('100ES15.7E2').
// A list-directed WRITE(u,*) ' ' ends every row and two more end the file.
bool write_columns(const OutJob& J, const std::string& path, int kind,
                   const std::vector<const double*>& cols, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  const size_t n = (size_t)J.nx * J.ny;
  (void)n;
  const int T = std::max(1, J.threads);
  const int band = 16;   // rows per task
  std::vector<std::string> text(T);
  bool ok = true;
  for (int k0 = 1; k0 <= J.ny && ok; k0 += band * T) {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
      th.emplace_back([&, t]() {
        std::string& o = text[t];
        o.clear();
        const int ka = k0 + t * band, kb = std::min(J.ny, ka + band - 1);
        for (int k = ka; k <= kb; ++k) {
          for (int j = 1; j <= J.nx; ++j) {
            const size_t c = (size_t)(j - 1) + (size_t)(k - 1) * J.nx;
            if (kind == 0) {
              ffmt::E(o, out_x_comp(J, j), 20, 12);
              ffmt::E(o, out_y_comp(J, k), 20, 12);
              for (const double* p : cols) ffmt::E(o, p[c], 20, 12);
            } else {
              ffmt::ES(o, out_x_comp(J, j), 15, 7, 2);
              ffmt::ES(o, out_y_comp(J, k), 15, 7, 2);
              for (const double* p : cols) ffmt::ES(o, p[c], 15, 7, 2);
            }
            o.push_back('\n');
          }
          o.append("  \n");
        }
      });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < T && ok; ++t)
      if (!text[t].empty() && std::fwrite(text[t].data(), 1, text[t].size(), f) != text[t].size())
        ok = false;
  }
  if (ok) ok = std::fputs("  \n  \n", f) >= 0;
  if (std::fclose(f) != 0) ok = false;
  if (!ok) err = "write failed: " + path;
  return ok;
}

// An ESRI grid as output_esri/output_max write it: the six header records
// ('(A,I5)' / '(A,F15.3)') and rows from north to south in '(2000ES12.3E3)',
// 2000 values per record.  `val(c)` gives the printed value of cell c.
template <class F>
bool write_esri(const OutJob& J, const std::string& path, F val, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::string o;
  o += "ncols ";
  ffmt::I(o, J.nx, 5);
  o += "\nnrows ";
  ffmt::I(o, J.ny, 5);
  o += "\nxllcorner ";
  ffmt::F(o, J.x0, 15, 3);
  o += "\nyllcorner ";
  ffmt::F(o, J.y0, 15, 3);
  o += "\ncellsize ";
  ffmt::F(o, J.cell_size, 15, 3);
  o += "\nNODATA_value ";
  ffmt::I(o, -9999, 5);
  o += "\n";
  bool ok = std::fwrite(o.data(), 1, o.size(), f) == o.size();
  // rows from north to south, formatted in bands by J.threads workers
  const int T = std::max(1, J.threads), band = 16;
  std::vector<std::string> text(T);
  for (int r0 = 0; r0 < J.ny && ok; r0 += band * T) {
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
      th.emplace_back([&, t]() {
        std::string& b = text[t];
        b.clear();
        const int ra = r0 + t * band, rb = std::min(J.ny, ra + band);
        for (int r = ra; r < rb; ++r) {
          const int k = J.ny - r;
          for (int j = 1; j <= J.nx; ++j) {
            ffmt::ES(b, val((size_t)(j - 1) + (size_t)(k - 1) * J.nx), 12, 3, 3);
            if (j % 2000 == 0 || j == J.nx) b.push_back('\n');
          }
        }
      });
    }
    for (auto& x : th) x.join();
    for (int t = 0; t < T && ok; ++t)
      if (!text[t].empty()) ok = std::fwrite(text[t].data(), 1, text[t].size(), f) == text[t].size();
  }
  if (std::fclose(f) != 0) ok = false;
  if (!ok) err = "write failed: " + path;
  return ok;
}

int run_out_job(const OutJob& J, std::string& err) {
  const size_t n = (size_t)J.nx * J.ny;
  auto P = [&](long off, int i) { return J.buf + (size_t)(off + i) * n; };
  const std::string idx = ffmt::lettera(J.idx - 1);
  if (J.cons) {
    std::vector<const double*> c;
    for (int i = 0; i < J.nv; ++i) c.push_back(P(J.q, i));
    if (!write_columns(J, J.run + "_" + idx + ".q_2d", 0, c, err)) return IMEX_EINVAL;
    if (J.erosion) {
      c.clear();
      for (int i = 0; i < J.ns; ++i) c.push_back(P(J.ers_c, i));
      if (!write_columns(J, J.run + "_erosion_" + idx + ".q_2d", 0, c, err)) return IMEX_EINVAL;
      c.clear();
      for (int i = 0; i < J.ns; ++i) c.push_back(P(J.erd_c, i));
      if (!write_columns(J, J.run + "_erodible_" + idx + ".q_2d", 0, c, err)) return IMEX_EINVAL;
    }
    if (J.settling) {
      c.clear();
      for (int i = 0; i < J.ns; ++i) c.push_back(P(J.dep_c, i));
      if (!write_columns(J, J.run + "_deposit_" + idx + ".q_2d", 0, c, err)) return IMEX_EINVAL;
    }
    if (J.topo) {
      c.assign(1, P(J.B_c, 0));
      if (!write_columns(J, J.run + "_B_" + idx + ".q_2d", 0, c, err)) return IMEX_EINVAL;
    }
  }
  if (J.phys) {
    std::vector<const double*> c;
    for (int i = 0; i < p2d_cols(J.ns); ++i) c.push_back(P(J.p2d, i));
    if (!write_columns(J, J.run + "_" + idx + ".p_2d", 1, c, err)) return IMEX_EINVAL;
  }
  if (J.esri) {
    const double* h = P(J.esr, 0);
    const double* T = P(J.esr, 1);
    if (!write_esri(J, J.run + "_" + idx + ".asc",
                    [&](size_t c) { return h[c] >= 1.0e-5 ? h[c] : -9999.0; }, err))
      return IMEX_EINVAL;
    if (!write_esri(J, J.run + "_T_" + idx + ".asc",
                    [&](size_t c) { return h[c] >= 1.0e-5 ? T[c] : -9999.0; }, err))
      return IMEX_EINVAL;
    auto tot = [&](long off, size_t c) {   // SUM(x(:,j,:),DIM=2)/(1-porosity)
      double s = 0.0;
      for (int i = 0; i < J.ns; ++i) s = s + P(off, i)[c];
      return s / (1.0 - J.porosity);
    };
    if (J.settling) {
      for (int i = 0; i < J.ns; ++i) {
        const double* d = P(J.dep_e, i);
        if (!write_esri(J, J.run + "_dep_" + ffmt::lettera(i + 1) + "_" + idx + ".asc",
                        [&](size_t c) { return d[c] > 0.0 ? d[c] : -9999.0; }, err))
          return IMEX_EINVAL;
      }
      if (!write_esri(J, J.run + "_depTot_" + idx + ".asc",
                      [&](size_t c) { const double v = tot(J.dep_e, c); return v > 0.0 ? v : -9999.0; },
                      err))
        return IMEX_EINVAL;
    }
    if (J.erosion) {
      for (int i = 0; i < J.ns; ++i) {
        const double* d = P(J.ers_e, i);
        if (!write_esri(J, J.run + "_ers_" + ffmt::lettera(i + 1) + "_" + idx + ".asc",
                        [&](size_t c) { return d[c] > 0.0 ? d[c] : -9999.0; }, err))
          return IMEX_EINVAL;
      }
      if (!write_esri(J, J.run + "_ersTot_" + idx + ".asc",
                      [&](size_t c) { const double v = tot(J.ers_e, c); return v > 0.0 ? v : -9999.0; },
                      err))
        return IMEX_EINVAL;
    }
  }
  if (J.maxf) {
    const double* hm = P(J.hmax, 0);
    if (!write_esri(J, J.run + "_max.asc",
                    [&](size_t c) { return hm[c] >= 1.0e-5 ? hm[c] : -9999.0; }, err))
      return IMEX_EINVAL;
  }
  return IMEX_OK;
}

template <int NS>
void launch_output_prep(ImexCtx* ctx, const OutputArgs& A) {
  const long long n = (long long)ctx->P.nx * ctx->P.ny;
  k_output_prep<NS><<<grid_1d(n, 128), 128, 0, ctx->stream>>>(ctx->P, A);
  ctx->launches += 1;
}

void output_prep(ImexCtx* ctx, const OutputArgs& A) {
  switch (ctx->ns) {
    case 1: launch_output_prep<1>(ctx, A); break;
    case 2: launch_output_prep<2>(ctx, A); break;
    case 3: launch_output_prep<3>(ctx, A); break;
    default: launch_output_prep<4>(ctx, A); break;
  }
}

}  // namespace

extern "C" {

int imex_format_edit(int kind, double value, int w, int d, int e, char* buf, int cap) {
  if (!buf || cap < 1 || w < 1 || w > 100 || d < 0 || d > 40 || e < 0 || e > 4) return -1;
  std::string o;
  switch (kind) {
    case 0: ffmt::E(o, value, w, d); break;
    case 1: ffmt::ES(o, value, w, d, e); break;
    case 2: ffmt::I(o, (long long)value, w); break;
    case 3: ffmt::F(o, value, w, d); break;
    default: return -1;
  }
  if ((int)o.size() >= cap) return -1;
  std::memcpy(buf, o.c_str(), o.size() + 1);
  return (int)o.size();
}

int imex_gpu_output_wait(ImexCtx* ctx) {
  if (!ctx) return IMEX_EINVAL;
  if (ctx->out_thread.joinable()) ctx->out_thread.join();
  ctx->out_pending = false;
  const int st = ctx->out_status;
  ctx->out_status = IMEX_OK;
  if (st != IMEX_OK) return fail(ctx, st, ctx->out_error);
  return IMEX_OK;
}

int imex_gpu_output(ImexCtx* ctx, const ImexOutputSpec* spec) {
  if (!ctx || !spec || !spec->run_name) return IMEX_EINVAL;
  int st = imex_gpu_output_wait(ctx);   // one job in flight: the staging buffer is reused
  if (st != IMEX_OK) return st;
  CK(cudaSetDevice(ctx->device));
  const DevParams& P = ctx->P;
  const ImexParams& hp = ctx->host_params;
  const int ns = ctx->ns, nv = P.nv;
  const size_t n = (size_t)P.nx * P.ny;
  OutJob J;
  J.run = spec->run_name;
  J.idx = spec->output_idx;
  J.nx = P.nx;
  J.ny = P.ny;
  J.ns = ns;
  J.nv = nv;
  J.threads = spec->threads > 0 ? spec->threads
                                 : std::max(1, (int)std::thread::hardware_concurrency());
  J.x0 = P.x0;
  J.y0 = P.y0;
  J.dx = P.dx;
  J.dy = P.dy;
  J.cell_size = hp.cell_size;
  J.porosity = hp.erodible_porosity;
  J.cons = spec->cons != 0;
  J.phys = spec->phys != 0;
  J.esri = spec->esri != 0;
  J.maxf = spec->max_grid != 0;
  J.erosion = hp.erosion_coeff > 0.0 && ctx->erosion;
  J.settling = hp.settling_flag && ctx->deposit;
  J.topo = hp.topo_change_flag && ctx->Bcent;
  if (J.maxf && !ctx->post_on)
    return fail(ctx, IMEX_EINVAL, "imex_gpu_output: the _max grid needs imex_gpu_post_init");
  // staged planes, in order
  long nplanes = 0;
  auto take = [&](long k) { const long o = nplanes; nplanes += k; return o; };
  if (J.cons) {
    J.q = take(nv);
    if (J.erosion) { J.ers_c = take(ns); J.erd_c = take(ns); }
    if (J.settling) J.dep_c = take(ns);
    if (J.topo) J.B_c = take(1);
  }
  if (J.phys) J.p2d = take(p2d_cols(ns));
  if (J.esri) {
    J.esr = take(2);
    if (J.settling) J.dep_e = take(ns);
    if (J.erosion) J.ers_e = take(ns);
  }
  if (J.maxf) J.hmax = take(1);
  if (nplanes == 0) return IMEX_OK;
  const size_t dev_need = ((J.phys ? p2d_cols(ns) : 0) + (J.esri ? 2 : 0)) * n;
  if (dev_need > ctx->out_dev_n) {
    if (ctx->out_dev) cudaFree(ctx->out_dev);
    ctx->out_dev = nullptr;
    ctx->out_dev_n = 0;
    CK(cudaMalloc((void**)&ctx->out_dev, dev_need * sizeof(double)));
    ctx->out_dev_n = dev_need;
  }
  const size_t host_need = (size_t)nplanes * n;
  if (host_need > ctx->out_host_n) {
    if (ctx->out_host) cudaFreeHost(ctx->out_host);
    ctx->out_host = nullptr;
    ctx->out_host_n = 0;
    CK(cudaMallocHost((void**)&ctx->out_host, host_need * sizeof(double)));
    ctx->out_host_n = host_need;
  }
  if (!ctx->out_ev) CK(cudaEventCreateWithFlags(&ctx->out_ev, cudaEventDisableTiming));
  double* p2d_dev = ctx->out_dev;
  double* esr_dev = ctx->out_dev + (J.phys ? (size_t)p2d_cols(ns) * n : 0);
  const size_t row = (size_t)P.nx * sizeof(double), pitch = (size_t)P.pitch * sizeof(double);
  auto stage_pitched = [&](long off, const double* src, int planes) -> cudaError_t {
    for (int i = 0; i < planes; ++i) {
      cudaError_t e = cudaMemcpy2DAsync(ctx->out_host + (size_t)(off + i) * n, row,
                                        src + (size_t)i * P.plane, pitch, row, P.ny,
                                        cudaMemcpyDeviceToHost, ctx->stream);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  OutputArgs A{};
  A.q = ctx->q;
  A.deposit = ctx->deposit;
  A.erosion = ctx->erosion;
  A.erodible = ctx->erodible;
  A.Bcent = ctx->Bcent;
  A.Bx = ctx->Bx;
  A.By = ctx->By;
  A.post = ctx->post;
  A.post_on = ctx->post_on ? 1 : 0;
  A.p2d = p2d_dev;
  A.esr = esr_dev;
  // the order of output_solution: ESRI's qp and the .q_2d zeroing of q, the
  // .q_2d planes, then the .p_2d values (zeroing DEPOSIT/EROSION), then the
  // ESRI planes
  if (J.cons || J.esri) {
    A.cons = J.cons;
    A.esri = J.esri;
    A.phys = 0;
    output_prep(ctx, A);
  }
  if (J.cons) {
    CK(stage_pitched(J.q, ctx->q, nv));
    if (J.erosion) {
      CK(stage_pitched(J.ers_c, ctx->erosion, ns));
      CK(stage_pitched(J.erd_c, ctx->erodible, ns));
    }
    if (J.settling) CK(stage_pitched(J.dep_c, ctx->deposit, ns));
    if (J.topo) CK(stage_pitched(J.B_c, ctx->Bcent, 1));
  }
  if (J.phys) {
    A.cons = 0;
    A.esri = 0;
    A.phys = 1;
    output_prep(ctx, A);
    CK(cudaMemcpyAsync(ctx->out_host + (size_t)J.p2d * n, p2d_dev,
                       (size_t)p2d_cols(ns) * n * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->stream));
  }
  if (J.esri) {
    CK(cudaMemcpyAsync(ctx->out_host + (size_t)J.esr * n, esr_dev, 2 * n * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->stream));
    if (J.settling) CK(stage_pitched(J.dep_e, ctx->deposit, ns));
    if (J.erosion) CK(stage_pitched(J.ers_e, ctx->erosion, ns));
  }
  if (J.maxf) CK(stage_pitched(J.hmax, ctx->post.hmax, 1));
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->out_ev, ctx->stream));
  J.buf = ctx->out_host;
  ctx->out_pending = true;
  ctx->out_status = IMEX_OK;
  ctx->out_error.clear();
  cudaEvent_t ev = ctx->out_ev;
  const int dev = ctx->device;
  ctx->out_thread = std::thread([ctx, J, ev, dev]() {
    cudaSetDevice(dev);
    cudaError_t e = cudaEventSynchronize(ev);
    if (e != cudaSuccess) {
      ctx->out_error = std::string("imex_gpu_output: ") + cudaGetErrorString(e);
      ctx->out_status = IMEX_ECUDA;
      return;
    }
    std::string err;
    const int st = run_out_job(J, err);
    if (st != IMEX_OK) {
      ctx->out_error = "imex_gpu_output: " + err;
      ctx->out_status = st;
    }
  });
  return IMEX_OK;
}

}  // extern "C"
