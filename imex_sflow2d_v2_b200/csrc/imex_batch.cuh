// imex_batch.cuh -- one time step of many independent runs (ensemble
// members) in one set of launches.
//
// Each phase of the step is one persistent kernel for all members: a fixed
// grid (a resident wave of blocks) walks a work list that the previous
// phase built on the device.  The mask pass walks every tile of every member
// and appends the tiles that hold a solve cell to the active-tile list; the
// flux, stage-2 and erosion passes walk only those tiles; the Newton
// iteration passes walk the members' Newton lists laid end to end.  The
// per-tile and per-cell work is the single-grid path's own device code
// (mask_tile, flux_tile, stage2_*_lane, stage2_post_cell,
// erosion_update_cell), so a member advances bit for bit as it does alone.
//
// The tile shape of the mask and flux passes is a template parameter: the
// ensemble's tuner times a real step with each shape and keeps the fastest
// (results do not depend on it).
#pragma once

#include "imex_kernels.cuh"

namespace imex {
inline namespace IMEX_TU_NS {

// A member as the batched kernels see it (device memory).
struct MemberDev {
  DevParams P;
  double* q;
  double* X;
  uint8_t* mask;
  const uint8_t* cellinfo;
  const double* release;
  const double *Bx, *By, *Bxx, *Bxy, *Byy, *gc, *dgc, *gcsx, *gcsy;
  const RingCell* ring;
  double *erodible, *deposit, *erosion, *Bcent;
  DevClock* clk;
  NewtonWork W;
  int tiles_x;        // tiles per row for the batch's tile shape
  int exchange;       // the erosion/deposition pass runs for this member
  long long tile0;    // first global tile index of the member
};

// The per-cell passes read a member's parameters from a copy in shared
// memory, refreshed when the block (or, in the list passes, the warp) moves
// to another member: read straight from global memory, the parameters the
// inner loops use add load latency and registers to every pass (measured
// 20-30% slower per pass than the single-grid kernels, whose parameters are
// a __grid_constant__ kernel argument).
__device__ __forceinline__ void stage_params(DevParams& dst, const DevParams& src, int tid,
                                             int nthreads) {
  static_assert(sizeof(DevParams) % 8 == 0 && alignof(DevParams) >= 8, "DevParams words");
  constexpr int W = (int)(sizeof(DevParams) / 8);
  const unsigned long long* a = reinterpret_cast<const unsigned long long*>(&src);
  unsigned long long* b = reinterpret_cast<unsigned long long*>(&dst);
  for (int i = tid; i < W; i += nthreads) b[i] = a[i];
}

// Position of global tile g: its member and its first cell (j0, k0).
struct TilePos {
  const MemberDev* D;
  int j0, k0;
};

__device__ __forceinline__ TilePos tile_pos(const MemberDev* __restrict__ M,
                                            const uint32_t* __restrict__ tile_member, long long g,
                                            int tx, int ty) {
  TilePos t;
  t.D = &M[tile_member[g]];
  const long long lt = g - t.D->tile0;
  t.j0 = (int)(lt % t.D->tiles_x) * tx;
  t.k0 = (int)(lt / t.D->tiles_x) * ty;
  return t;
}

// Clock work of all members: one thread per member.
__global__ void kb_step_begin(MemberDev* M, int n, unsigned int* n_active) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) *n_active = 0;
  if (m < n) {
    step_begin(M[m].clk, M[m].P.max_dt, 1);
    nw_reset(M[m].clk);
  }
}

__global__ void kb_dt_clip(MemberDev* M, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) dt_clip(M[m].clk, 1);
}

__global__ void kb_step_end(MemberDev* M, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) step_end(M[m].clk);
}

// check_solve of every tile of every member; tiles with a solve cell go to
// the active list.
template <class TS>
__global__ void __launch_bounds__(256)
    kb_mask(const MemberDev* __restrict__ M, const uint32_t* __restrict__ tile_member,
            long long n_tiles, uint32_t* __restrict__ active, unsigned int* n_active) {
  __shared__ uint8_t s0[TS::SH][TS::SW];
  __shared__ uint8_t s1[TS::SH][TS::SW];
  for (long long g = blockIdx.x; g < n_tiles; g += gridDim.x) {
    const TilePos t = tile_pos(M, tile_member, g, TS::TX, TS::TY);
    const MemberDev& D = *t.D;
    const bool any = mask_tile<TS>(D.P, D.q, D.release, D.cellinfo, D.clk->t, D.mask, D.clk, 0,
                                   t.j0, t.k0, s0, s1);
    if (any && threadIdx.x == 0) active[atomicAdd(n_active, 1u)] = (uint32_t)g;
  }
}

// The flux pass stages a member's parameters in shared memory too, when the
// copy leaves the blocks per SM unchanged (kb_flux_smem: the bytes of one
// block).
template <int NS, class TS>
__host__ __device__ constexpr bool flux_stages_params() {
  return (size_t)flux_min_blocks<NS, TS>() * (sizeof(FluxShared<NS, TS>) + sizeof(DevParams) + 1024) <=
         (size_t)228 * 1024;
}
template <int NS, class TS>
__host__ __device__ constexpr size_t kb_flux_smem() {
  return sizeof(FluxShared<NS, TS>) + (flux_stages_params<NS, TS>() ? sizeof(DevParams) : 0);
}

// Stage 1 and the CFL minimum of the active tiles.
template <int NS, class TS>
__global__ void __launch_bounds__(TS::THREADS, (flux_min_blocks<NS, TS>()))
    kb_flux(const MemberDev* __restrict__ M, const uint32_t* __restrict__ tile_member,
            const uint32_t* __restrict__ active, const unsigned int* __restrict__ n_active) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FluxShared<NS, TS>& S = *reinterpret_cast<FluxShared<NS, TS>*>(smem_raw);
  DevParams& sP = *reinterpret_cast<DevParams*>(smem_raw + sizeof(FluxShared<NS, TS>));
  const unsigned int n = *n_active;
  const MemberDev* cur = nullptr;
  for (unsigned int a = blockIdx.x; a < n; a += gridDim.x) {
    const TilePos t = tile_pos(M, tile_member, active[a], TS::TX, TS::TY);
    const MemberDev& D = *t.D;
    if constexpr (flux_stages_params<NS, TS>()) {
      if (t.D != cur) {
        __syncthreads();
        stage_params(sP, D.P, threadIdx.x, blockDim.x);
        __syncthreads();
        cur = t.D;
      }
      flux_tile<NS, TS>(sP, D.q, D.mask, D.cellinfo, D.Bx, D.By, D.Bxx, D.Bxy, D.Byy, D.gc,
                        D.dgc, D.gcsx, D.gcsy, D.ring, D.clk, D.X, t.j0, t.k0, S);
    } else {
      flux_tile<NS, TS>(D.P, D.q, D.mask, D.cellinfo, D.Bx, D.By, D.Bxx, D.Bxy, D.Byy, D.gc,
                        D.dgc, D.gcsx, D.gcsy, D.ring, D.clk, D.X, t.j0, t.k0, S);
    }
  }
}

// Stage 2 up to Newton iteration 1 on the cells of the active tiles (tiles
// of tx x ty cells, walked in warp-sized runs of consecutive cells).
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_FIRST_MINB)
    kb_stage2_first(const MemberDev* __restrict__ M, const uint32_t* __restrict__ tile_member,
                    const uint32_t* __restrict__ active, const unsigned int* __restrict__ n_active,
                    int tx, int ty) {
  __shared__ DevParams sP;
  const unsigned int n = *n_active;
  const MemberDev* cur = nullptr;
  for (unsigned int a = blockIdx.x; a < n; a += gridDim.x) {
    const TilePos t = tile_pos(M, tile_member, active[a], tx, ty);
    const MemberDev& D = *t.D;
    if (t.D != cur) {
      __syncthreads();
      stage_params(sP, D.P, threadIdx.x, blockDim.x);
      __syncthreads();
      cur = t.D;
    }
    const double dt = D.clk->dt;
    unsigned long long cells = 0, it_sum = 0, maxit = 0;
    for (int base = 0; base < tx * ty; base += blockDim.x) {
      const int e = base + threadIdx.x;
      const int j = t.j0 + e % tx, k = t.k0 + e / tx;
      const bool valid = e < tx * ty && j < sP.nx && k < sP.ny;
      const size_t c = valid ? (size_t)k * sP.pitch + j : 0;
      stage2_first_lane<NS>(sP, D.q, D.X, D.mask, D.Bx, D.By, D.Bxx, D.Bxy, D.Byy, D.gc, D.W,
                            D.clk, dt, valid, c, cells, it_sum, maxit);
    }
    newton_flush_stats(D.clk, cells, it_sum, 0, maxit);
  }
}

// The members' lists `which` laid end to end, each padded to a multiple of
// 32 entries so that a warp never spans two members: off[m] is member m's
// first slot, off[n] the total.  One block.
__global__ void __launch_bounds__(1024)
    kb_list_offsets(const MemberDev* __restrict__ M, int n, int which,
                    unsigned long long* __restrict__ off) {
  __shared__ unsigned long long warp_sum[32];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int m0 = threadIdx.x * per;
  unsigned long long s = 0;
  for (int m = m0; m < m0 + per && m < n; ++m)
    s += ((unsigned long long)M[m].clk->nw_count[which] + 31ULL) & ~31ULL;
  // inclusive scan of s over the block
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long x = s;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sum[w] = x;
  __syncthreads();
  if (w == 0) {
    unsigned long long v = lane < (int)(blockDim.x >> 5) ? warp_sum[lane] : 0ULL;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    warp_sum[lane] = v;
  }
  __syncthreads();
  unsigned long long excl = x - s + (w > 0 ? warp_sum[w - 1] : 0ULL);
  for (int m = m0; m < m0 + per && m < n; ++m) {
    off[m] = excl;
    excl += ((unsigned long long)M[m].clk->nw_count[which] + 31ULL) & ~31ULL;
  }
  if (threadIdx.x == blockDim.x - 1) off[n] = excl;
}

// Member of slot e of the laid-out lists (off ascending, n+1 entries).
__device__ __forceinline__ int list_member(const unsigned long long* __restrict__ off, int n,
                                           unsigned long long e) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Newton iteration nl_iter (2 or 3) over the members' lists nl_iter-2.
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    kb_stage2_iter(const MemberDev* __restrict__ M, int n, const unsigned long long* __restrict__ off,
                   int nl_iter) {
  __shared__ DevParams sP[STAGE2_THREADS / 32];
  DevParams& wP = sP[threadIdx.x >> 5];
  int cur = -1;
  const unsigned long long total = off[n];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
       base < total; base += stride) {
    const int m = list_member(off, n, base);
    const MemberDev& D = M[m];
    if (m != cur) {
      __syncwarp();
      stage_params(wP, D.P, threadIdx.x & 31, 32);
      __syncwarp();
      cur = m;
    }
    const long long e = (long long)(base - off[m]) + (threadIdx.x & 31);
    const bool valid = e < (long long)D.clk->nw_count[nl_iter - 2];
    unsigned long long it_sum = 0, maxit = 0, trials = 0;
    stage2_iter_lane<NS>(wP, D.q, D.Bx, D.By, D.W, D.clk, D.clk->dt, nl_iter, valid, e, it_sum,
                         maxit, trials);
    newton_flush_stats(D.clk, 0, it_sum, trials, maxit);
  }
}

// Iterations 4..100 over the members' lists 2.
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    kb_stage2_tail(const MemberDev* __restrict__ M, int n, const unsigned long long* __restrict__ off) {
  __shared__ DevParams sP[STAGE2_THREADS / 32];
  DevParams& wP = sP[threadIdx.x >> 5];
  int cur = -1;
  const unsigned long long total = off[n];
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
       base < total; base += stride) {
    const int m = list_member(off, n, base);
    const MemberDev& D = M[m];
    if (m != cur) {
      __syncwarp();
      stage_params(wP, D.P, threadIdx.x & 31, 32);
      __syncwarp();
      cur = m;
    }
    const long long e = (long long)(base - off[m]) + (threadIdx.x & 31);
    const bool valid = e < (long long)D.clk->nw_count[2];
    unsigned long long it_sum = 0, maxit = 0, trials = 0;
    stage2_tail_lane<NS>(wP, D.q, D.Bx, D.By, D.W, D.clk, D.clk->dt, valid, e, it_sum, maxit,
                         trials);
    newton_flush_stats(D.clk, 0, it_sum, trials, maxit);
  }
}

// Sign guard and assembly on the solve cells of the active tiles.
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS)
    kb_stage2_post(const MemberDev* __restrict__ M, const uint32_t* __restrict__ tile_member,
                   const uint32_t* __restrict__ active, const unsigned int* __restrict__ n_active,
                   int tx, int ty) {
  __shared__ DevParams sP;
  const unsigned int n = *n_active;
  const MemberDev* cur = nullptr;
  for (unsigned int a = blockIdx.x; a < n; a += gridDim.x) {
    const TilePos t = tile_pos(M, tile_member, active[a], tx, ty);
    const MemberDev& D = *t.D;
    if (t.D != cur) {
      __syncthreads();
      stage_params(sP, D.P, threadIdx.x, blockDim.x);
      __syncthreads();
      cur = t.D;
    }
    for (int e = threadIdx.x; e < tx * ty; e += blockDim.x) {
      const int j = t.j0 + e % tx, k = t.k0 + e / tx;
      if (j >= sP.nx || k >= sP.ny || !D.mask[(size_t)k * sP.pitch + j]) continue;
      stage2_post_cell<NS>(sP, D.q, D.cellinfo, D.W, D.clk, j, k);
    }
  }
}

// Erosion/deposition on the solve cells of the active tiles of the members
// that exchange mass with the bed.
template <int NS>
__global__ void __launch_bounds__(128, IMEX_EROSION_MINB)
    kb_erosion(const MemberDev* __restrict__ M, const uint32_t* __restrict__ tile_member,
               const uint32_t* __restrict__ active, const unsigned int* __restrict__ n_active,
               int tx, int ty) {
  __shared__ DevParams sP;
  const unsigned int n = *n_active;
  const MemberDev* cur = nullptr;
  for (unsigned int a = blockIdx.x; a < n; a += gridDim.x) {
    const TilePos t = tile_pos(M, tile_member, active[a], tx, ty);
    const MemberDev& D = *t.D;
    if (!D.exchange) continue;
    if (t.D != cur) {
      __syncthreads();
      stage_params(sP, D.P, threadIdx.x, blockDim.x);
      __syncthreads();
      cur = t.D;
    }
    const double dt = D.clk->dt;
    for (int e = threadIdx.x; e < tx * ty; e += blockDim.x) {
      const int j = t.j0 + e % tx, k = t.k0 + e / tx;
      if (j >= sP.nx || k >= sP.ny || !D.mask[(size_t)k * sP.pitch + j]) continue;
      erosion_update_cell<NS>(sP, D.q, D.Bx, D.By, D.erodible, D.deposit, D.erosion, D.Bcent,
                              D.clk, dt, j, k);
    }
  }
}

}  // namespace IMEX_TU_NS
}  // namespace imex
