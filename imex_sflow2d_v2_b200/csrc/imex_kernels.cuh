// imex_kernels.cuh -- the per-step kernels of the IMEX_SfloW2D time step.
//
//   k_mask      check_solve: wet/source seed, n_RK=2 four-neighbour dilation in
//               shared memory, inlet-interior removal (src/solver_2d.f90:666-857)
//   k_flux      one tile per block: physical states of the tile and a 2-cell
//               halo in shared memory, MUSCL faces with the reference's
//               boundary/inlet rules, local speeds, Kurganov-Tadmor fluxes,
//               divergence, explicit terms and the CFL minimum
//               (timestep + RK stage 1: src/solver_2d.f90:872-1005,2614-3918)
//   k_stage2_*  RK stage 2: semi-implicit terms, Newton with line search and
//               complex-step Jacobian (one pass per Newton iteration over the
//               cells still iterating), assembly checks
//               (src/solver_2d.f90:1105-1628, 1660-2365)
//   k_erosion   the erosion/deposition update per cell
//               (src/solver_2d.f90:2380-2595)
//
// Data layout: structure-of-arrays planes, plane v of q at q + v*plane,
// element (j,k) (0-based) at k*pitch + j.
#pragma once

#include <type_traits>

#include <cuda.h>   // CUtensorMap (the type only; maps are encoded by the host)

#include "imex_device.cuh"
#include "imex_mlp.cuh"

namespace imex {
inline namespace IMEX_TU_NS {

constexpr int HALO = 2;

// A tile of TXv x TYv cells: its shared-memory extent with the 2-cell halo,
// its interface counts and the threads of a flux block (one per cell, plus
// one warp, so that every cell keeps its own thread between the x and y
// phases of k_flux).
template <int TXv, int TYv>
struct TileShape {
  static constexpr int TX = TXv, TY = TYv;
  static constexpr int SW = TX + 2 * HALO;    // shared tile width
  static constexpr int SH = TY + 2 * HALO;    // shared tile height
  static constexpr int NXI = (TX + 1) * TY;   // x-interfaces per tile
  static constexpr int NYI = TX * (TY + 1);   // y-interfaces per tile
  static constexpr int THREADS = TX * TY + 32;
};
using Shape32x8 = TileShape<32, 8>;    // the single-grid path's tiles
using Shape16x16 = TileShape<16, 16>;
using Shape32x4 = TileShape<32, 4>;

constexpr int TX = Shape32x8::TX;
constexpr int TY = Shape32x8::TY;
constexpr int SW = Shape32x8::SW;
constexpr int SH = Shape32x8::SH;
constexpr int FLUX_THREADS = Shape32x8::THREADS;
constexpr int NXI = Shape32x8::NXI;
constexpr int NYI = Shape32x8::NYI;

// Minimum resident blocks per SM asked of ptxas for the flux and per-cell
// kernels (their register budget); tuning knobs, set with -D at build time.
// The Newton list passes run at 128 registers (4 blocks of 128): 7.34 ms
// per step at 4096^2 against 7.63 at 96 registers and 7.79 at 80.
#ifndef IMEX_STAGE2_MINB
#define IMEX_STAGE2_MINB 4
#endif
#ifndef IMEX_EROSION_MINB
#define IMEX_EROSION_MINB 8
#endif

// Device clock shared by the step kernels (graph-replayable).
struct DevClock {
  double t, dt, dt_old, dt_old_old, t_end, t_output;
  unsigned long long dtmin_bits;  // running CFL minimum (positive doubles)
  unsigned int error_mask;
  int pad_;
  unsigned long long first_error;  // (cell index << 8) | code, min over cells
  unsigned long long newton_cells, newton_iters, lnsrch_trials, newton_maxit;
  unsigned long long hist[16];
  unsigned long long solve_cells;
  unsigned long long steps;
  unsigned int nw_count[4];  // cells appended to the stage-2 Newton lists
                             // ([3]: the warm-start list)
  unsigned long long harvest_n;      // training pairs written so far
  unsigned long long warm_fallback;  // warm starts redone from q_si
  unsigned int nw_fb;                // cells in the warm-start fallback list
  int pad2_;
};

IMEX_HD double x_stag(const DevParams& P, int J) { return P.x0 + (double)(J - 1) * P.dx; }
IMEX_HD double y_stag(const DevParams& P, int K) { return P.y0 + (double)(K - 1) * P.dy; }
IMEX_HD double x_comp(const DevParams& P, int J) { return 0.5 * (x_stag(P, J) + x_stag(P, J + 1)); }
IMEX_HD double y_comp(const DevParams& P, int K) { return 0.5 * (y_stag(P, K) + y_stag(P, K + 1)); }

__device__ __forceinline__ void record_error(DevClock* clk, int code, long long cell) {
  atomicOr(&clk->error_mask, 1u << code);
  unsigned long long key = ((unsigned long long)cell << 8) | (unsigned long long)code;
  atomicMin(&clk->first_error, key);
}

__device__ const RingCell* find_ring(const RingCell* ring, int n, long long idx) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    long long v = ring[mid].idx;
    if (v == idx) return &ring[mid];
    if (v < idx) lo = mid + 1; else hi = mid - 1;
  }
  return nullptr;
}

// ================================================================= k_mask
// check_solve(.FALSE.) for n_RK = 2 on the tile whose first cell is
// (j0, k0): the wet/source seed of the tile and a 2-cell halo, two 4-point
// dilations, the border rows and the inlet-interior removal.  Returns, to
// every thread of the block, whether any cell of the tile is solved.
template <class TS>
__device__ __forceinline__ bool mask_tile(const DevParams& P, const double* __restrict__ q1,
                                          const double* __restrict__ release_time,
                                          const uint8_t* __restrict__ cellinfo, double t,
                                          uint8_t* __restrict__ mask, DevClock* clkw,
                                          int solve_all, int j0, int k0,
                                          uint8_t (*s0)[TS::SW], uint8_t (*s1)[TS::SW]) {
  constexpr int SWt = TS::SW, SHt = TS::SH, TXt = TS::TX, TYt = TS::TY;
  const int nx = P.nx, ny = P.ny;
  for (int e = threadIdx.x; e < SWt * SHt; e += blockDim.x) {
    int lx = e % SWt, ly = e / SWt;
    int j = j0 + lx - HALO, k = k0 + ly - HALO;
    uint8_t m = 0;
    if (j >= 0 && j < nx && k >= 0 && k < ny) {
      bool border = (j == 0 || j == nx - 1 || k == 0 || k == ny - 1);
      if (border || solve_all) {
        m = 1;
      } else {
        size_t c = (size_t)k * P.pitch + j;
        bool rel = P.has_release_time ? (release_time[c] <= t) : (0.0 <= t);
        if (q1[c] > 0.0 && rel) m = 1;
        if (P.radial_source_flag && (cellinfo[(size_t)k * nx + j] & CI_SRC_MASK) == 2) m = 1;
      }
    }
    s0[ly][lx] = m;
  }
  __syncthreads();
  // first dilation on the tile plus a 1-cell ring
  for (int e = threadIdx.x; e < SWt * SHt; e += blockDim.x) {
    int lx = e % SWt, ly = e / SWt;
    int j = j0 + lx - HALO, k = k0 + ly - HALO;
    uint8_t m = s0[ly][lx];
    if (lx >= 1 && lx < SWt - 1 && ly >= 1 && ly < SHt - 1 && j >= 1 && j < nx - 1 && k >= 1 &&
        k < ny - 1)
      m = m | s0[ly][lx - 1] | s0[ly][lx + 1] | s0[ly - 1][lx] | s0[ly + 1][lx];
    s1[ly][lx] = m;
  }
  __syncthreads();
  int cnt = 0;
  for (int e = threadIdx.x; e < TXt * TYt; e += blockDim.x) {
    int lx = e % TXt + HALO, ly = e / TXt + HALO;
    int j = j0 + lx - HALO, k = k0 + ly - HALO;
    if (j >= nx || k >= ny) continue;
    uint8_t m = s1[ly][lx];
    if (j >= 1 && j < nx - 1 && k >= 1 && k < ny - 1)
      m = m | s1[ly][lx - 1] | s1[ly][lx + 1] | s1[ly - 1][lx] | s1[ly + 1][lx];
    if (P.radial_source_flag && (cellinfo[(size_t)k * nx + j] & CI_SRC_MASK) == 1) m = 0;
    mask[(size_t)k * P.pitch + j] = m;
    cnt += m;
  }
  const bool any = __syncthreads_or(cnt) != 0;
  // solve-cell count
  for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(&clkw->solve_cells, (unsigned long long)cnt);
  return any;
}

__global__ void __launch_bounds__(256) k_mask(const __grid_constant__ DevParams Pp, const double* __restrict__ q1,
                                              const double* __restrict__ release_time,
                                              const uint8_t* __restrict__ cellinfo,
                                              const DevClock* clk, uint8_t* __restrict__ mask,
                                              DevClock* clkw, int solve_all) {
  __shared__ uint8_t s0[SH][SW];
  __shared__ uint8_t s1[SH][SW];
  mask_tile<Shape32x8>(Pp, q1, release_time, cellinfo, clk->t, mask, clkw, solve_all,
                       blockIdx.x * TX, blockIdx.y * TY, s0, s1);
}

// ------------------------------------------------------ TMA tile loads
// One bulk tensor copy per tile (cp.async.bulk.tensor, this GPU's memory
// only, no multicast) completing on a shared-memory mbarrier.  The wait is
// bounded: past the limit the caller records IMEX_ETIMEOUT (never expected).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
// makes the barrier's initialisation visible to the copy engine's proxy
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
constexpr int TMA_WAIT_LIMIT = 1 << 22;   // try_wait polls (seconds at most)
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t phase) {
  for (int it = 0; it < TMA_WAIT_LIMIT; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

// k_mask over the tile rows [ty0, ty0 + gridDim.y): one band of a step whose
// state arrives from the host band by band (imex_gpu_advance_host).
__global__ void __launch_bounds__(256) k_mask_rows(const __grid_constant__ DevParams Pp,
                                                   const double* __restrict__ q1,
                                                   const double* __restrict__ release_time,
                                                   const uint8_t* __restrict__ cellinfo,
                                                   const DevClock* clk, uint8_t* __restrict__ mask,
                                                   DevClock* clkw, int ty0) {
  __shared__ uint8_t s0[SH][SW];
  __shared__ uint8_t s1[SH][SW];
  mask_tile<Shape32x8>(Pp, q1, release_time, cellinfo, clk->t, mask, clkw, 0, blockIdx.x * TX,
                       (blockIdx.y + ty0) * TY, s0, s1);
}

// ================================================================== faces
// Shared tile of physical states: qps[v][ly][lx]; info_s[ly][lx] holds the
// cellinfo bits plus bit 7 = solve mask.
template <int NS, class TS = Shape32x8>
struct Tile {
  double qp[6 + NS][TS::SH][TS::SW];
  uint8_t info[TS::SH][TS::SW];
};

// Face states of one cell in one direction: W/E (dir 1) or S/N (dir 2).
// `stage` selects the RK-stage arrays' view of never-solved inlet-interior
// neighbours (all zero) instead of the module qp view (zero with T_ambient).
template <int NS, class TS>
IMEX_FLAT void cell_faces(const DevParams& P, const Tile<NS, TS>& T, int lx, int ly, int j, int k,
                           int dir, bool stage, double time, const RingCell* ring,
                           double* Fm, double* Fp) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const uint8_t inf = T.info[ly][lx];
  const int scell = inf & CI_SRC_MASK;
  const bool rad = P.radial_source_flag != 0;
  const bool sE = inf & CI_E, sW = inf & CI_W, sS = inf & CI_S, sN = inf & CI_N;
  double sb[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) sb[i] = 0.0;
  if (rad && scell == 2) {
    const RingCell* rc = find_ring(ring, P.n_ring, (long long)k * P.nx + j);
    if (rc) {
      int w = sE ? 0 : (sW ? 1 : (sS ? 2 : 3));
      eval_source_bdry<NS>(P, time, rc->vx[w], rc->vy[w], sb);
    }
  }
  auto nb = [&](int v, int d) -> double {
    int cx = (dir == 1) ? lx + d : lx;
    int cy = (dir == 1) ? ly : ly + d;
    if (stage && (T.info[cy][cx] & CI_SRC_MASK) == 1 && rad) return 0.0;
    return T.qp[v][cy][cx];
  };
  const int J = j + 1, K = k + 1;  // Fortran indices
  const int n = (dir == 1) ? P.nx : P.ny;
  const int I = (dir == 1) ? J : K;
  const double dh = (dir == 1) ? P.dx2 : P.dy2;
  const double one_by_d = (dir == 1) ? P.one_by_dx : P.one_by_dy;
  auto comp = [&](int m) { return (dir == 1) ? x_comp(P, m) : y_comp(P, m); };
  auto stag = [&](int m) { return (dir == 1) ? x_stag(P, m) : y_stag(P, m); };
  const int* flagm = (dir == 1) ? P.bcW_flag : P.bcS_flag;
  const int* flagp = (dir == 1) ? P.bcE_flag : P.bcN_flag;
  const double* valm = (dir == 1) ? P.bcW_val : P.bcS_val;
  const double* valp = (dir == 1) ? P.bcE_val : P.bcN_val;
  // inlet-ring corrections apply to the x direction through sE/sW and to the
  // y direction through sS/sN; border inlet cells (lateral source) use the
  // inlet state as the Dirichlet value in x only.
  const bool ring_m = rad && scell == 2 && ((dir == 1) ? (!sE && sW) : (sS));
  const bool ring_p = rad && scell == 2 && ((dir == 1) ? sE : (!sS && sN));
  const bool border_src = (dir == 1) && scell == 2;
  // stencil abscissae after the n_vars loop
  double z1, z2 = comp(I), z3;
  if (I == 1) {
    z1 = stag(1);
    z3 = comp(2);
  } else if (I == n) {
    z1 = comp(n - 1);
    z3 = stag(n + 1);
  } else {
    z1 = ring_m ? stag(I) : comp(I - 1);
    z3 = ring_p ? stag(I + 1) : comp(I + 1);
  }
  const double rc_d = P.reconstr_coeff * dh;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double v2 = nb(i, 0), slope;
    if (I == 1) {
      if (border_src) {
        slope = limit(sb[i], v2, nb(i, 1), z1, z2, z3, P.limiter[i], P.theta);
      } else if (flagm[i] == 0) {
        slope = limit(valm[i], v2, nb(i, 1), z1, z2, z3, P.limiter[i], P.theta);
      } else if (flagm[i] == 1) {
        slope = valm[i];
      } else {
        slope = (nb(i, 1) - nb(i, 0)) * one_by_d;
      }
    } else if (I == n) {
      if (border_src) {
        slope = limit(nb(i, -1), v2, sb[i], z1, z2, z3, P.limiter[i], P.theta);
      } else if (flagp[i] == 0) {
        slope = limit(nb(i, -1), v2, valp[i], z1, z2, z3, P.limiter[i], P.theta);
      } else if (flagp[i] == 1) {
        slope = valp[i];
      } else {
        slope = (nb(i, 0) - nb(i, -1)) * one_by_d;
      }
    } else {
      double v1 = ring_m ? sb[i] : nb(i, -1);
      double v3 = ring_p ? sb[i] : nb(i, 1);
      slope = limit(v1, v2, v3, z1, z2, z3, P.limiter[i], P.theta);
    }
    double dq = rc_d * slope;
    double fm = v2 - dq, fp = v2 + dq;
    const int ivel = (dir == 1) ? 1 : 2;  // hu clamp in x, hv clamp in y
    if (I == 1) {
      if (border_src) fm = sb[i];
      else if (flagm[i] == 0) fm = valm[i];
      else if (i == ivel) fm = fmin_f(fm, 0.0);
    }
    if (I == n) {
      if (border_src) fp = sb[i];
      else if (flagp[i] == 0) fp = valp[i];
      else if (i == ivel) fp = fmax_f(fp, 0.0);
    }
    Fm[i] = fm;
    Fp[i] = fp;
  }
  // u and v with the limiters of hu and hv
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const int i = NV + a;
    double zz1 = z1, zz3 = z3;
    if (dir == 1 && a == 1 && rad && scell == 2 && I > 1 && I < n && !sE && sN && !sS &&
        K > 1 && K < P.ny)
      zz3 = y_stag(P, K + 1);  // x_stencil(3)=y_stag(k+1), src/solver_2d.f90:3616
    double v2 = nb(i, 0), v1, v3;
    if (I == 1) {
      v1 = (Fm[0] <= 0.0) ? 0.0 : Fm[1 + a] / Fm[0];
      v3 = nb(i, 1);
    } else if (I == n) {
      v1 = nb(i, -1);
      v3 = (Fp[0] <= 0.0) ? 0.0 : Fp[1 + a] / Fp[0];
    } else {
      v1 = ring_m ? sb[i] : nb(i, -1);
      v3 = ring_p ? sb[i] : nb(i, 1);
    }
    double slope = limit(v1, v2, v3, zz1, z2, zz3, P.limiter[i], P.theta);
    double dq = rc_d * slope;
    Fm[i] = v2 - dq;
    Fp[i] = v2 + dq;
    if (I == 1) Fm[i] = v1;
    else if (I == n) Fp[i] = v3;
  }
  if (I > 1 && I < n) {
    if (ring_p) {
#pragma unroll
      for (int i = 0; i < NP; ++i) Fp[i] = sb[i];
    } else if (ring_m) {
#pragma unroll
      for (int i = 0; i < NP; ++i) Fm[i] = sb[i];
    }
  }
}

// One interface: left/lower state from cell a, right/upper from cell b.
// Writes the KT flux H (n_vars) and max(|a+|,|a-|) for the CFL.
// Limited MUSCL increments of one direction, precomputed once per cell for
// the cells whose faces need none of cell_faces' special rules: not on the
// domain border in that direction, not an inlet cell, no inlet-interior
// neighbour in that direction (so the stage and timestep views agree).
// There the faces are qp -/+ rc_d*limit(...) for every variable, exactly the
// operations of cell_faces.  Indexed [ly - 1][lx - 1] of the shared tile:
// x faces use rows 2..9 and columns 1..34, y faces rows 1..10, columns 2..33.
template <int NS, class TS = Shape32x8>
struct SlopeTile {
  double dq[6 + NS][TS::TY + 2][TS::TX + 2];
  uint8_t ok[TS::TY + 2][TS::TX + 2];
};

template <int NS, class TS>
__device__ __forceinline__ void precompute_slopes(const DevParams& P, const Tile<NS, TS>& T,
                                                  SlopeTile<NS, TS>& D, int dir, int j0, int k0,
                                                  const uint8_t* __restrict__ mask) {
  constexpr int NP = 6 + NS, TX = TS::TX, TY = TS::TY;
  const int nx = P.nx, ny = P.ny;
  const bool rad = P.radial_source_flag != 0;
  const int rw = (dir == 1) ? TX + 2 : TX, rh = (dir == 1) ? TY : TY + 2;
  for (int e = threadIdx.x; e < rw * rh; e += blockDim.x) {
    const int lx = (dir == 1) ? 1 + e % rw : HALO + e % rw;
    const int ly = (dir == 1) ? HALO + e / rw : 1 + e / rw;
    const int j = j0 + lx - HALO, k = k0 + ly - HALO;
    uint8_t ok = 0;
    const int I = (dir == 1) ? j + 1 : k + 1, n = (dir == 1) ? nx : ny;
    if (j >= 0 && j < nx && k >= 0 && k < ny && I > 1 && I < n) {
      const uint8_t inf = T.info[ly][lx];
      const int dx_ = (dir == 1) ? 1 : 0, dy_ = (dir == 1) ? 0 : 1;
      // an active interface on either side: the cell or a neighbour is solved
      const bool used = (inf & 128) || (T.info[ly - dy_][lx - dx_] & 128) ||
                        (T.info[ly + dy_][lx + dx_] & 128);
      const bool plain = !(rad && (inf & CI_SRC_MASK) != 0) &&
                         !(rad && (T.info[ly - dy_][lx - dx_] & CI_SRC_MASK) == 1) &&
                         !(rad && (T.info[ly + dy_][lx + dx_] & CI_SRC_MASK) == 1);
      if (used && plain) {
        const double dh = (dir == 1) ? P.dx2 : P.dy2;
        const double rc_d = P.reconstr_coeff * dh;
        const double z1 = (dir == 1) ? x_comp(P, I - 1) : y_comp(P, I - 1);
        const double z2 = (dir == 1) ? x_comp(P, I) : y_comp(P, I);
        const double z3 = (dir == 1) ? x_comp(P, I + 1) : y_comp(P, I + 1);
        const double dz = z3 - z2;
        const bool uniform = (dz == z2 - z1) && (z3 > z2) && (z2 > z1);
#pragma unroll 1
        for (int i = 0; i < NP; ++i) {
          const double v1 = T.qp[i][ly - dy_][lx - dx_], v2 = T.qp[i][ly][lx],
                       v3 = T.qp[i][ly + dy_][lx + dx_];
          const double lim = (uniform && P.limiter[i] == 1)
                                 ? minmod_uniform(v1, v2, v3, dz, z1, z2, z3, P.theta)
                                 : limit(v1, v2, v3, z1, z2, z3, P.limiter[i], P.theta);
          D.dq[i][ly - 1][lx - 1] = rc_d * lim;
        }
        ok = 1;
      }
    }
    D.ok[ly - 1][lx - 1] = ok;
  }
}

template <int NS, class TS>
IMEX_FLAT void interface_flux(const DevParams& P, const Tile<NS, TS>& T, int dir, int la_x,
                               int la_y, int ja, int ka, bool a_in, bool b_in, double gcf,
                               bool stage, double time, const RingCell* ring, double* H,
                               double& amax_flux, double& aneg_out, double& apos_out,
                               const SlopeTile<NS, TS>* D = nullptr) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const int lb_x = (dir == 1) ? la_x + 1 : la_x, lb_y = (dir == 1) ? la_y : la_y + 1;
  const int jb = (dir == 1) ? ja + 1 : ja, kb = (dir == 1) ? ka : ka + 1;
  double QL[NP], QR[NP], tmpm[NP], tmpp[NP];
  const bool rad = P.radial_source_flag != 0;
  const uint8_t ia = a_in ? T.info[la_y][la_x] : 0, ib = b_in ? T.info[lb_y][lb_x] : 0;
  const bool a_int = rad && a_in && (ia & CI_SRC_MASK) == 1;
  const bool b_int = rad && b_in && (ib & CI_SRC_MASK) == 1;
  const uint8_t flag_b_m = (dir == 1) ? CI_W : CI_S;  // b's inlet lies on its minus side
  const uint8_t flag_a_p = (dir == 1) ? CI_E : CI_N;
  // reconstruction of the sides that need it, through one call site
  const bool comp_a = a_in && (!b_in || !a_int);
  const bool comp_b = b_in && (!a_in || !b_int);
#pragma unroll 1
  for (int side = 0; side < 2; ++side) {
    if (!(side == 0 ? comp_a : comp_b)) continue;
    const int sx = side ? lb_x : la_x, sy = side ? lb_y : la_y;
    if (D && stage && D->ok[sy - 1][sx - 1]) {
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const double v2 = T.qp[i][sy][sx], dq = D->dq[i][sy - 1][sx - 1];
        tmpm[i] = v2 - dq;
        tmpp[i] = v2 + dq;
      }
    } else {
      cell_faces<NS>(P, T, sx, sy, side ? jb : ja, side ? kb : ka, dir, stage, time, ring,
                     tmpm, tmpp);
    }
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      if (side == 0) QL[i] = tmpp[i];   // a's plus face
      else QR[i] = tmpm[i];             // b's minus face
    }
  }
  if (!a_in) {  // domain boundary on the minus side: both states from b's minus face
#pragma unroll
    for (int i = 0; i < NP; ++i) QL[i] = QR[i];
  } else if (!b_in) {
#pragma unroll
    for (int i = 0; i < NP; ++i) QR[i] = QL[i];
  } else {
    const bool have_a = comp_a, have_b = comp_b;
    if (a_int) {
      // never solved: only the ring copy of src/solver_2d.f90:3768-3771 fills it
      bool copy = have_b && (ib & flag_b_m) && (ib & CI_SRC_MASK) == 2 &&
                  ((dir == 1) ? !(ib & CI_E) : true);
      if (dir == 2) copy = have_b && (ib & CI_S) && (ib & CI_SRC_MASK) == 2;
#pragma unroll
      for (int i = 0; i < NP; ++i) QL[i] = copy ? QR[i] : 0.0;
    }
    if (b_int) {
      bool copy = have_a && (ia & flag_a_p) && (ia & CI_SRC_MASK) == 2;
      if (dir == 2) copy = have_a && (ia & CI_N) && !(ia & CI_S) && (ia & CI_SRC_MASK) == 2;
#pragma unroll
      for (int i = 0; i < NP; ++i) QR[i] = copy ? QL[i] : 0.0;
    }
  }
  double cL[NV], cR[NV];
  Mixt mL, mR;
  face_qc_mixt<NS>(P, QL, cL, mL);
  face_qc_mixt<NS>(P, QR, cR, mR);
  double lmin, lmax, rmin, rmax;
  local_speeds<NS>(P, QL, mL, gcf, dir, lmin, lmax);
  local_speeds<NS>(P, QR, mR, gcf, dir, rmin, rmax);
  double aN = fmin_f(fmin_f(lmin, rmin), 0.0);
  double aP = fmax_f(fmax_f(lmax, rmax), 0.0);
  aneg_out = aN;
  apos_out = aP;
  amax_flux = fmax_f(aP, -aN);
  double fL[NV], fR[NV];
  eval_fluxes<NS>(P, cL, QL, mL, gcf, dir, fL);
  eval_fluxes<NS>(P, cR, QR, mR, gcf, dir, fR);
  if (aN == aP) {
#pragma unroll
    for (int i = 0; i < NV; ++i) H[i] = 0.0;
  } else {
    double coef = (aP * aN) / (aP - aN);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double avg = (aP * fL[i] - aN * fR[i]) / (aP - aN);
      H[i] = avg + coef * (cR[i] - cL[i]);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) s += H[4 + i];
  if (dir == 1) {
    if (s / H[0] >= 1.0) {
      double r = 0.0;
#pragma unroll
      for (int i = 0; i < NS; ++i) r += H[4 + i] / H[0];
#pragma unroll
      for (int i = 0; i < NS; ++i) H[4 + i] = H[4 + i] / r;
    }
    if (QL[1] == 0.0 && QR[1] == 0.0) {
      H[0] = 0.0;
#pragma unroll
      for (int i = 3; i < NV; ++i) H[i] = 0.0;
    }
  } else {
    if (s / H[0] > 1.0) {
      double r = s / H[0];
#pragma unroll
      for (int i = 0; i < NS; ++i) H[4 + i] = H[4 + i] / r;
    }
    if (cL[2] == 0.0 && cR[2] == 0.0) {
      H[0] = 0.0;
#pragma unroll
      for (int i = 3; i < NV; ++i) H[i] = 0.0;
    }
  }
}

// ================================================================= k_flux
// Shared memory: Tile<NS> + slopes + one direction's interface fluxes and
// CFL speeds at a time (the x ones are reduced into each cell's registers
// before the y phase overwrites them).
template <int NS, class TS = Shape32x8>
struct FluxShared {
  Tile<NS, TS> tile;
  union {
    SlopeTile<NS, TS> slopes;
    // the tile's conserved variables as one TMA box (k_flux_tma), read
    // before the slopes are first written
    alignas(128) double stage[4 + NS][TS::SH][TS::SW];
  };
  union {
    double Hx[4 + NS][TS::TY][TS::TX + 1];
    double Hy[4 + NS][TS::TY + 1][TS::TX];
  } H;
  union {
    double ax[TS::TY][TS::TX + 1];
    double ay[TS::TY + 1][TS::TX];
  } A;
  double dtmin[TS::THREADS / 32];
  unsigned long long tma_bar;   // mbarrier of the TMA box
};
static_assert(Shape32x8::THREADS == 288, "k_flux blocks of 288 threads for 32x8 tiles");

// Blocks of k_flux per SM: 3 where three blocks' shared memory fits the SM
// (228 KB, 1 KB reserved per block; n_s <= 3), else 2.  At n_s = 3 three
// blocks at 72 registers measured 9.5 ms per step at 4096^2 against 10.9 at
// two blocks of 96.
// Other tile shapes keep the register budget of three 288-thread blocks
// (864 threads per SM) and fit as many blocks as shared memory allows.
template <int NS, class TS = Shape32x8>
__host__ __device__ constexpr int flux_min_blocks() {
#ifdef IMEX_FLUX_MINB
  return IMEX_FLUX_MINB;
#else
  return std::is_same<TS, Shape32x8>::value
             ? ((3 * (sizeof(FluxShared<NS, TS>) + 1024) <= 228 * 1024) ? 3 : 2)
             : ((864 / TS::THREADS) < (int)(228 * 1024 / (sizeof(FluxShared<NS, TS>) + 1024))
                    ? (864 / TS::THREADS)
                    : (int)(228 * 1024 / (sizeof(FluxShared<NS, TS>) + 1024)));
#endif
}

// k_cfl_tiles: the tile and both directions' CFL speeds.
template <int NS>
struct CflShared {
  Tile<NS> tile;
  double ax[TY][TX + 1];
  double ay[TY + 1][TX];
  double dtmin[FLUX_THREADS / 32];
};

// Stage 1 and the CFL minimum on the tile whose first cell is (j0, k0).
template <int NS, class TS>
__device__ __forceinline__ void flux_tile(const DevParams& P, const double* __restrict__ q,
                                          const uint8_t* __restrict__ mask,
                                          const uint8_t* __restrict__ cellinfo,
                                          const double* __restrict__ Bx,
                                          const double* __restrict__ By,
                                          const double* __restrict__ Bxx,
                                          const double* __restrict__ Bxy,
                                          const double* __restrict__ Byy,
                                          const double* __restrict__ gc,
                                          const double* __restrict__ dgc,
                                          const double* __restrict__ gcsx,
                                          const double* __restrict__ gcsy,
                                          const RingCell* __restrict__ ring, DevClock* clk,
                                          double* __restrict__ X, int j0, int k0,
                                          FluxShared<NS, TS>& S,
                                          const CUtensorMap* qmap = nullptr) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  constexpr int TX = TS::TX, TY = TS::TY, SW = TS::SW, SH = TS::SH, NXI = TS::NXI,
                NYI = TS::NYI;
  const int nx = P.nx, ny = P.ny;
  const double time = clk->t;
  // any solve cell in the tile?
  int any = 0;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    int j = j0 + e % TX, k = k0 + e / TX;
    if (j < nx && k < ny && mask[(size_t)k * P.pitch + j]) any = 1;
  }
  if (!__syncthreads_or(any)) return;
  // With a tensor map of q, the tile's n_v planes (halo included, zeros
  // outside the grid) arrive as one TMA box in the staging area
  const bool staged = qmap != nullptr;
  if (staged) {
    static_assert(sizeof(S.stage) == (size_t)(4 + NS) * SH * SW * sizeof(double), "box size");
    if (threadIdx.x == 0) {
      mbar_init(&S.tma_bar, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&S.tma_bar, (uint32_t)sizeof(S.stage));
      // x = j0 - 2 is even: 16-byte aligned for 8-byte elements
      tma_load_3d(&S.stage[0][0][0], qmap, j0 - HALO, k0 - HALO, 0, &S.tma_bar);
    }
    const bool arrived = mbar_wait_bounded(&S.tma_bar, 0);
    if (__syncthreads_or(!arrived)) {
      // never expected: record it, wait (bounded) for the copy, and leave
      if (threadIdx.x == 0) record_error(clk, 7, (long long)k0 * nx + j0);
      mbar_wait_bounded(&S.tma_bar, 0);
      return;
    }
  }
  // physical states of the tile + halo
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
        // inlet interior: never solved, holds its allocation value
#pragma unroll
        for (int i = 0; i < NP; ++i) qpv[i] = 0.0;
        qpv[3] = P.T_ambient;
      } else {
#pragma unroll
        for (int i = 0; i < NV; ++i) qc[i] = staged ? S.stage[i][ly][lx] : q[c + (size_t)i * P.plane];
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
  // interfaces: x faces (e < NXI), then y faces, one interface per thread;
  // each direction's slopes are precomputed once per cell first
  const RingCell* rg = ring;
  // this thread's cell (one per thread): the x part of the divergence and
  // the x CFL dt, taken before the y phase reuses the flux arrays
  double dX[NV], dtx = P.max_dt;
  for (int pdir = 1; pdir <= 2; ++pdir) {
  precompute_slopes<NS>(P, S.tile, S.slopes, pdir, j0, k0, mask);
  __syncthreads();
  for (int e = (pdir == 1 ? 0 : NXI) + threadIdx.x; e < (pdir == 1 ? NXI : NXI + NYI);
       e += blockDim.x) {
    const int dir = (e < NXI) ? 1 : 2;
    int jj, kk, ja, ka, ia_x, ia_y;
    bool a_in, b_in, sa, sb_;
    if (dir == 1) {
      // interface between cells (j0+jj-1) and (j0+jj) in row k0+kk
      jj = e % (TX + 1);
      kk = e / (TX + 1);
      ja = j0 + jj - 1;
      ka = k0 + kk;
      ia_x = jj - 1 + HALO;
      ia_y = kk + HALO;
    } else {
      const int e2 = e - NXI;
      jj = e2 % TX;
      kk = e2 / TX;
      ja = j0 + jj;
      ka = k0 + kk - 1;
      ia_x = jj + HALO;
      ia_y = kk - 1 + HALO;
    }
    double& a_slot = (dir == 1) ? S.A.ax[kk][jj] : S.A.ay[kk][jj];
    const bool exists = (dir == 1) ? !(ka >= ny || ja + 1 > nx) : !(ja >= nx || ka + 1 > ny);
    // a direction of one cell has no fluxes and no speeds: the reference
    // skips its speeds, fluxes and divergence term (src/solver_2d.f90:
    // 2667-2681, 3946-4001), and its zero-initialised speed arrays give no
    // CFL limit there
    const bool flat = (dir == 1) ? nx == 1 : ny == 1;
    if (!exists || flat) { a_slot = 0.0; continue; }
    if (dir == 1) {
      a_in = ja >= 0;
      b_in = ja + 1 < nx;
      sa = a_in && (S.tile.info[ia_y][ia_x] & 128);
      sb_ = b_in && (S.tile.info[ia_y][ia_x + 1] & 128);
    } else {
      a_in = ka >= 0;
      b_in = ka + 1 < ny;
      sa = a_in && (S.tile.info[ia_y][ia_x] & 128);
      sb_ = b_in && (S.tile.info[ia_y + 1][ia_x] & 128);
    }
    if (!(sa || sb_)) { a_slot = 0.0; continue; }
    double gcf = 1.0;
    if (P.slope_correction_flag)
      gcf = (dir == 1) ? gcsx[(size_t)ka * (nx + 1) + (ja + 1)] : gcsy[(size_t)(ka + 1) * nx + ja];
    // CFL from the timestep view when an inlet-interior cell is in the stencil
    bool dual = false;
    if (P.radial_source_flag) {
      for (int d = -1; d <= 2; ++d) {
        const int cx = (dir == 1) ? ia_x + d : ia_x, cy = (dir == 1) ? ia_y : ia_y + d;
        const int cg = (dir == 1) ? ja + d : ka + d, cn = (dir == 1) ? nx : ny;
        if (cg >= 0 && cg < cn && (S.tile.info[cy][cx] & CI_SRC_MASK) == 1) dual = true;
      }
    }
    double H[NV], amax = 0.0, aN, aP;
#pragma unroll 1
    for (int pass = 0; pass < (dual ? 2 : 1); ++pass) {
      double Hp[NV];
      interface_flux<NS>(P, S.tile, dir, ia_x, ia_y, ja, ka, a_in, b_in, gcf, pass == 0, time, rg,
                         Hp, amax, aN, aP, &S.slopes);
      if (pass == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) H[i] = Hp[i];
      }
    }
    if (dir == 1) {
#pragma unroll
      for (int i = 0; i < NV; ++i) S.H.Hx[i][kk][jj] = H[i];
    } else {
#pragma unroll
      for (int i = 0; i < NV; ++i) S.H.Hy[i][kk][jj] = H[i];
    }
    a_slot = amax;
  }
  __syncthreads();
  if (pdir == 1 && threadIdx.x < TX * TY) {
    const int jj = threadIdx.x % TX, kk = threadIdx.x / TX;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double d = 0.0;
      if (nx > 1) d = d + (S.H.Hx[i][kk][jj + 1] - S.H.Hx[i][kk][jj]) * P.one_by_dx;
      dX[i] = d;
    }
    const double max_a = fmax_f(S.A.ax[kk][jj], S.A.ax[kk][jj + 1]);
    dtx = (max_a > 0.0) ? P.cfl * P.dx / max_a : P.max_dt;
  }
  }
  // cells: divergence, explicit terms, CFL
  double dtl = P.max_dt;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    int jj = e % TX, kk = e / TX;
    int j = j0 + jj, k = k0 + kk;
    if (j >= nx || k >= ny) continue;
    int lx = jj + HALO, ly = kk + HALO;
    if (!(S.tile.info[ly][lx] & 128)) continue;
    size_t c = (size_t)k * P.pitch + j;
    double qpv[NP], ex[NV];
#pragma unroll
    for (int i = 0; i < NP; ++i) qpv[i] = S.tile.qp[i][ly][lx];
    double bx = Bx[c], by = By[c];
    double bxx = 0.0, bxy = 0.0, byy = 0.0, gcf = 1.0, dg = 0.0;
    if (P.curvature_term_flag) {
      bxx = Bxx[c];
      bxy = Bxy[c];
      byy = Byy[c];
    }
    if (P.slope_correction_flag) {
      gcf = gc[c];
      dg = dgc[c];
    }
    eval_expl_terms<NS>(P, bx, by, bxx, bxy, byy, gcf, dg, qpv, ex);
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      double d = dX[i];
      if (ny > 1) d = d + (S.H.Hy[i][kk + 1][jj] - S.H.Hy[i][kk][jj]) * P.one_by_dy;
      X[c + (size_t)i * P.plane] = d - ex[i];
    }
    const double max_a = fmax_f(S.A.ay[kk][jj], S.A.ay[kk + 1][jj]);
    double dty = (max_a > 0.0) ? P.cfl * P.dy / max_a : dtl;
    dtl = fmin_f(dtl, fmin_f(dtx, dty));
  }
  // block minimum, then a global atomic min on the bits of the positive double
  for (int off = 16; off > 0; off >>= 1) dtl = fmin_f(dtl, __shfl_down_sync(0xffffffffu, dtl, off));
  if ((threadIdx.x & 31) == 0) S.dtmin[threadIdx.x >> 5] = dtl;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = S.dtmin[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin_f(m, S.dtmin[w]);
    // a speed of +inf gives a cell dt of +0.0, which the reference's MIN
    // keeps; the block minimum is never negative and NaN is filtered by
    // fmin_f, so the ordered-bits atomicMin sees only non-negative doubles
    if (m >= 0.0 && m < P.max_dt)
      atomicMin(&clk->dtmin_bits, (unsigned long long)__double_as_longlong(m));
  }
}

template <int NS>
__global__ void __launch_bounds__(FLUX_THREADS, flux_min_blocks<NS>())
    k_flux(const __grid_constant__ DevParams Pp, const double* __restrict__ q, const uint8_t* __restrict__ mask,
           const uint8_t* __restrict__ cellinfo, const double* __restrict__ Bx,
           const double* __restrict__ By, const double* __restrict__ Bxx,
           const double* __restrict__ Bxy, const double* __restrict__ Byy,
           const double* __restrict__ gc, const double* __restrict__ dgc,
           const double* __restrict__ gcsx, const double* __restrict__ gcsy,
           const RingCell* __restrict__ ring, DevClock* clk, double* __restrict__ X) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FluxShared<NS>& S = *reinterpret_cast<FluxShared<NS>*>(smem_raw);
  flux_tile<NS, Shape32x8>(Pp, q, mask, cellinfo, Bx, By, Bxx, Bxy, Byy, gc, dgc, gcsx, gcsy, ring,
                           clk, X, blockIdx.x * TX, blockIdx.y * TY, S);
}

// k_flux with the tile's q planes loaded by one TMA box (qmap: a tensor map
// of q, dims {nx, ny, n_v}, box {SW, SH, n_v}, zero fill outside the grid).
template <int NS>
__global__ void __launch_bounds__(FLUX_THREADS, flux_min_blocks<NS>())
    k_flux_tma(const __grid_constant__ DevParams Pp, const __grid_constant__ CUtensorMap qmap,
               const double* __restrict__ q, const uint8_t* __restrict__ mask,
               const uint8_t* __restrict__ cellinfo, const double* __restrict__ Bx,
               const double* __restrict__ By, const double* __restrict__ Bxx,
               const double* __restrict__ Bxy, const double* __restrict__ Byy,
               const double* __restrict__ gc, const double* __restrict__ dgc,
               const double* __restrict__ gcsx, const double* __restrict__ gcsy,
               const RingCell* __restrict__ ring, DevClock* clk, double* __restrict__ X) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FluxShared<NS>& S = *reinterpret_cast<FluxShared<NS>*>(smem_raw);
  flux_tile<NS, Shape32x8>(Pp, q, mask, cellinfo, Bx, By, Bxx, Bxy, Byy, gc, dgc, gcsx, gcsy, ring,
                           clk, X, blockIdx.x * TX, blockIdx.y * TY, S, &qmap);
}

// k_flux_tma over the tile rows [ty0, ty0 + gridDim.y) (imex_gpu_advance_host).
template <int NS>
__global__ void __launch_bounds__(FLUX_THREADS, flux_min_blocks<NS>())
    k_flux_tma_rows(const __grid_constant__ DevParams Pp, const __grid_constant__ CUtensorMap qmap,
                    const double* __restrict__ q, const uint8_t* __restrict__ mask,
                    const uint8_t* __restrict__ cellinfo, const double* __restrict__ Bx,
                    const double* __restrict__ By, const double* __restrict__ Bxx,
                    const double* __restrict__ Bxy, const double* __restrict__ Byy,
                    const double* __restrict__ gc, const double* __restrict__ dgc,
                    const double* __restrict__ gcsx, const double* __restrict__ gcsy,
                    const RingCell* __restrict__ ring, DevClock* clk, double* __restrict__ X,
                    int ty0) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FluxShared<NS>& S = *reinterpret_cast<FluxShared<NS>*>(smem_raw);
  flux_tile<NS, Shape32x8>(Pp, q, mask, cellinfo, Bx, By, Bxx, Bxy, Byy, gc, dgc, gcsx, gcsy, ring,
                           clk, X, blockIdx.x * TX, (blockIdx.y + ty0) * TY, S, &qmap);
}

// k_flux over the tile rows [ty0, ty0 + gridDim.y) (imex_gpu_advance_host).
template <int NS>
__global__ void __launch_bounds__(FLUX_THREADS, flux_min_blocks<NS>())
    k_flux_rows(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                const uint8_t* __restrict__ mask, const uint8_t* __restrict__ cellinfo,
                const double* __restrict__ Bx, const double* __restrict__ By,
                const double* __restrict__ Bxx, const double* __restrict__ Bxy,
                const double* __restrict__ Byy, const double* __restrict__ gc,
                const double* __restrict__ dgc, const double* __restrict__ gcsx,
                const double* __restrict__ gcsy, const RingCell* __restrict__ ring, DevClock* clk,
                double* __restrict__ X, int ty0) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FluxShared<NS>& S = *reinterpret_cast<FluxShared<NS>*>(smem_raw);
  flux_tile<NS, Shape32x8>(Pp, q, mask, cellinfo, Bx, By, Bxx, Bxy, Byy, gc, dgc, gcsx, gcsy, ring,
                           clk, X, blockIdx.x * TX, (blockIdx.y + ty0) * TY, S);
}

// =============================================================== Newton
// solve_rk_step (src/solver_2d.f90:1660-1994) for a_diag = 1 (stage 2 of the
// n_RK = 2 tableau), cut at its iteration boundaries: newton_start (scaling
// and the test before the first iteration), newton_iter1 (the first
// iteration, a full step) and newton_iterk (every later iteration, with the
// line search).  The stage-2 passes below run one iteration per pass over a
// compacted list of the cells still iterating; each cell goes through
// exactly the operation sequence of one uninterrupted solve_rk_step.
constexpr int NEWTON_MAX_IT = 100;
constexpr double NEWTON_TOLF = 1.0e-10, NEWTON_STPMX = 100.0;

#ifndef IMEX_EVAL_FN
#define IMEX_EVAL_FN IMEX_FLAT
#endif
template <int NS>
IMEX_EVAL_FN void eval_f(const DevParams& P, const double* qj, const double* qj_old,
                       const double* Rj, double bx, double by, double dt, double* f,
                       double& scal_f) {
  constexpr int NV = 4 + NS;
  double nh2, nh3;
  implicit_terms_r<NS>(P, bx, by, qj, nh2, nh3);
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double nh = (i == 1) ? nh2 : ((i == 2) ? nh3 : 0.0);
    double R = Rj[i] - 1.0 * nh;
    double fi = qj[i] - qj_old[i] + dt * R;
    f[i] = 1.0 * fi;
  }
  double d = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) d += f[i] * f[i];
  scal_f = 0.5 * d;
}

// Jacobian columns 2,3 by complex step (src/solver_2d.f90:2300-2365) and the
// Newton direction: explicit rows diagonal, 2x2 Cramer on rows/cols 2,3
// (src/solver_2d.f90:1879-1901).
template <int NS, bool COLS_TOGETHER = false>
IMEX_FLAT void newton_direction(const DevParams& P, double bx, double by, double dt,
                                              const double* qj_org, const double* qj_rel,
                                              const double* rt, double* dd, double* J2,
                                              double* J3) {
  constexpr int NV = 4 + NS;
  CPrefix<NS> pre;
  {
    cplx qc[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) qc[m] = mulr(C(qj_rel[m], 0.0), qj_org[m]);
    implicit_prefix_c<NS>(P, qc, pre);
  }
  auto column = [&](int col) {
    cplx qc[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) qc[m] = mulr(C(qj_rel[m], (m == col) ? P.hstep : 0.0), qj_org[m]);
    cplx nh2, nh3;
    implicit_terms_c<NS>(P, bx, by, qc, pre, nh2, nh3);
#pragma unroll
    for (int r = 0; r < NV; ++r) {
      double nim = (r == 1) ? nh2.im : ((r == 2) ? nh3.im : 0.0);
      double jac = 1.0 * nim * P.one_by_h;
      double l0 = (r == col) ? 1.0 * (col == 1 ? qj_org[1] : qj_org[2]) : 0.0;
      double v = l0 - dt * 1.0 * jac;
      if (col == 1) J2[r] = v;
      else J3[r] = v;
    }
  };
  // the two columns one after the other, or (COLS_TOGETHER) unrolled, so
  // that the scheduler may interleave their independent chains
  if constexpr (COLS_TOGETHER) {
#pragma unroll
    for (int col = 1; col <= 2; ++col) column(col);
  } else {
#pragma unroll 1
    for (int col = 1; col <= 2; ++col) column(col);
  }
  double d1[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) d1[i] = (i == 1 || i == 2) ? 0.0 : rt[i] / (1.0 * qj_org[i]);
  double d2a = rt[1], d2b = rt[2];
  {
    double s = 0.0, s2 = 0.0;
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (i != 1 && i != 2) s += d1[i] * 0.0;
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (i != 1 && i != 2) s2 += d1[i] * 0.0;
    d2a = d2a - s;
    d2b = d2b - s2;
  }
  double s11 = J2[1], s21 = J2[2], s12 = J3[1], s22 = J3[2];
  double inv_det = 1.0 / (s11 * s22 - s21 * s12);
  double sol0 = (d2a * s22 - d2b * s12) * inv_det;
  double sol1 = (s11 * d2b - s21 * d2a) * inv_det;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    if (i == 1) dd[i] = -sol0 + 0.0;
    else if (i == 2) dd[i] = -sol1 + 0.0;
    else dd[i] = 0.0 + (-d1[i]);
  }
}

// The exit tests at the end of an iteration (src/solver_2d.f90:1964-1988).
template <int NS>
__device__ __forceinline__ bool newton_converged(const double* rt, const double* qj_rel,
                                                 const double* x_old) {
  constexpr int NV = 4 + NS;
  double mx = fabs(rt[0]);
#pragma unroll
  for (int i = 1; i < NV; ++i) mx = fmax_f(mx, fabs(rt[i]));
  if (mx < NEWTON_TOLF) return true;
  // m3 = MAX over i of |qj_rel - x_old| / MAX(|qj_rel|, 1) < EPS.  MAX skips
  // NaN quotients (all NaN: NaN, and the test fails), so the test holds when
  // some quotient is a number and every such quotient is below EPS; each
  // comparison of a rounded quotient is taken without the division where
  // its answer is certain (rel_change_below).
  bool any = false, below = true;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    const double d = fabs(qj_rel[i] - x_old[i]), s = fmax_f(fabs(qj_rel[i]), 1.0);
    if (isnan(d) || (isinf(d) && isinf(s))) continue;   // the quotient is NaN
    any = true;
    below = below & rel_change_below(d, s, EPS);
  }
  return any && below;
}

// Scaling (src/solver_2d.f90:1786-1798); the residual test before the first
// Jacobian.  True: q already satisfies TOLF (exit with nl_iter = 1).
template <int NS>
__device__ __forceinline__ void newton_scale(const double* qj, double* qj_org) {
  constexpr int NV = 4 + NS;
#pragma unroll
  for (int i = 0; i < NV; ++i) qj_org[i] = fmax_f(fabs(qj[i]), 1.0e-3);
}

template <int NS>
__device__ bool newton_start(const DevParams& P, const double* qj, const double* qj_old,
                             const double* Rj, double bx, double by, double dt,
                             const double* qj_org, double* qj_rel, double* rt, double& scal_f) {
  constexpr int NV = 4 + NS;
#pragma unroll
  for (int i = 0; i < NV; ++i) qj_rel[i] = qj[i] / qj_org[i];
  eval_f<NS>(P, qj, qj_old, Rj, bx, by, dt, rt, scal_f);
  double mx = fabs(rt[0]);
#pragma unroll
  for (int i = 1; i < NV; ++i) mx = fmax_f(mx, fabs(rt[i]));
  return mx < NEWTON_TOLF;
}

// Iteration 1: full Newton step, no line search.  qj receives the iterate.
template <int NS>
__device__ bool newton_iter1(const DevParams& P, double* qj, const double* qj_old,
                             const double* Rj, double bx, double by, double dt,
                             const double* qj_org, double* qj_rel, double* rt, double& scal_f) {
  constexpr int NV = 4 + NS;
  double dd[NV], J2[NV], J3[NV], x_old[NV];
  newton_direction<NS>(P, bx, by, dt, qj_org, qj_rel, rt, dd, J2, J3);
#pragma unroll
  for (int i = 0; i < NV; ++i) x_old[i] = qj_rel[i];
#pragma unroll
  for (int i = 0; i < NV; ++i) qj_rel[i] = x_old[i] + dd[i];
#pragma unroll
  for (int i = 0; i < NV; ++i) qj[i] = qj_rel[i] * qj_org[i];
  eval_f<NS>(P, qj, qj_old, Rj, bx, by, dt, rt, scal_f);
#pragma unroll
  for (int i = 0; i < NV; ++i) qj[i] = qj_rel[i] * qj_org[i];
  return newton_converged<NS>(rt, qj_rel, x_old);
}

// The residual at the iterate when the previous line search put the old
// iterate back (rare); true when it already meets TOLF.  Inlined: as a call
// the iteration pass measured 14.2 against 10.3 ms at 4096^2 (the arrays it
// takes then live in local memory for the whole pass).
#ifndef IMEX_RESTART_FN
#define IMEX_RESTART_FN __device__ __forceinline__
#endif
template <int NS>
IMEX_RESTART_FN bool newton_restart(const DevParams& P, double* qj, const double* qj_old,
                                    const double* Rj, double bx, double by, double dt,
                                    const double* qj_org, const double* qj_rel, double* rt,
                                    double& scal_f) {
  constexpr int NV = 4 + NS;
#pragma unroll
  for (int i = 0; i < NV; ++i) qj[i] = qj_rel[i] * qj_org[i];
  eval_f<NS>(P, qj, qj_old, Rj, bx, by, dt, rt, scal_f);
  double mx = fabs(rt[0]);
#pragma unroll
  for (int i = 1; i < NV; ++i) mx = fmax_f(mx, fabs(rt[i]));
  return mx < NEWTON_TOLF;
}

// Iterations 2..100: residual at the iterate, Newton direction and lnsrch
// (src/solver_2d.f90:1815-1824, 1929-1962, 2019-2224).  The reference
// evaluates the residual at the start of every iteration; it equals the one
// left by the previous iteration unless that iteration's line search put the
// old iterate back (alam < alamin or the trial cap), leaving the residual of
// its last trial: `stale` marks that case and the residual is evaluated
// again (the loop only continues after such a restore when the relative
// step is NaN).  Every backtrack after the first halves alam: the cubic
// model's value is clamped to <= alam/2 and then maxed with alam/2.  The
// trials are capped at 4096; the cap exits like alam < alamin.
template <int NS>
IMEX_FLAT bool newton_iterk(const DevParams& P, double* qj, const double* qj_old,
                                          const double* Rj, double bx, double by, double dt,
                                          const double* qj_org, double* qj_rel, double* rt,
                                          double& scal_f, long long& trials, bool& stale) {
  constexpr int NV = 4 + NS;
  if (stale) {
    stale = false;
    if (newton_restart<NS>(P, qj, qj_old, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f)) return true;
  }
  double dd[NV], J2[NV], J3[NV], x_old[NV];
  // the later iterations evaluate the Jacobian columns side by side (0.3 ms
  // per step less at 4096^2 than one column at a time)
  newton_direction<NS, true>(P, bx, by, dt, qj_org, qj_rel, rt, dd, J2, J3);
#pragma unroll
  for (int i = 0; i < NV; ++i) x_old[i] = qj_rel[i];
  const double scal_f_old = scal_f;
  double sdot = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) sdot += qj_rel[i] * qj_rel[i];
  double stpmax = NEWTON_STPMX * fmax_f(sqrt(sdot), (double)NV);
  double grad[NV];
#pragma unroll
  for (int c = 0; c < NV; ++c) {
    double s = 0.0;
#pragma unroll
    for (int r = 0; r < NV; ++r) {
      double L;
      if (c == 1) L = J2[r];
      else if (c == 2) L = J3[r];
      else L = (r == c) ? 1.0 * qj_org[c] : 0.0;
      s += rt[r] * L;
    }
    grad[c] = s;
  }
  // NORM2(dd) > stpmax scales the step.  The scaled sum below ends with
  // scale = MAX|dd| and ssq <= NV (each term at most 1) up to a few
  // roundings, so its result is below 3*MAX|dd| for NV <= 8; when that bound
  // is already below stpmax (finite), the norm cannot exceed it and is not
  // evaluated.  A NaN component gives a NaN norm and no scaling either way.
  static_assert(NV <= 8, "the norm bound 3*MAX|dd| holds for up to 8 components");
  double dmax = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) dmax = fmax_f(dmax, fabs(dd[i]));
  if (!(3.0 * dmax < stpmax)) {
    double scale = 0.0, ssq = 0.0;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      if (dd[i] != 0.0) {
        double ax = fabs(dd[i]);
        if (scale < ax) {
          double val = scale / ax;
          ssq = 1.0 + ssq * val * val;
          scale = ax;
        } else {
          double val = ax / scale;
          ssq = ssq + val * val;
        }
      }
    }
    double dabs = scale * sqrt(ssq);
    if (dabs > stpmax) {
#pragma unroll
      for (int i = 0; i < NV; ++i) dd[i] = dd[i] * stpmax / dabs;
    }
  }
  double slope = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) slope += grad[i] * dd[i];
  double mx = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double r = fabs(dd[i]) / fmax_f(fabs(x_old[i]), 1.0);
    mx = (i == 0) ? r : fmax_f(mx, r);
  }
  double alamin = EPS / mx;
  bool xfin = true;
#pragma unroll
  for (int i = 0; i < NV; ++i) xfin &= isfinite(x_old[i]);
  if (alamin == 0.0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) qj_rel[i] = x_old[i];
  } else {
    // Rows other than 2, 3 carry no implicit term: eval_f's sum of f^2
    // taken over them alone, in eval_f's order, cannot exceed the full sum
    // (rounded addition of a term >= 0 never decreases a sum, and rounding
    // is monotone).  When that partial half-sum already exceeds
    // 0.9*scal_f_old the trial fails whatever the implicit terms are, and
    // the implicit terms are not evaluated.  Only for trials whose failure
    // is all that matters: not trial 0 and not alam = 1 (their scal_f sets
    // the next alam), and with a finite old iterate (then the residual left
    // by the last trial is never read: a search that puts the old iterate
    // back ends the iteration as converged).
    //
    // After the first backtrack every alam is half the previous one,
    // whatever a trial's outcome, so two consecutive trials' partial sums
    // are evaluated side by side (independent chains) and their outcomes
    // then taken in order, as one trial after the other.
    auto partial_half_sum = [&](double al) {
      double d = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        if (i == 1 || i == 2) continue;
        const double qt = (x_old[i] + al * dd[i]) * qj_org[i];
        const double R = Rj[i] - 1.0 * 0.0;
        const double fi = qt - qj_old[i] + dt * R;
        const double f = 1.0 * fi;
        d += f * f;
      }
      return 0.5 * d;
    };
    const double sf_thr = 0.9 * scal_f_old;
    double alam = 1.0;
    int trial = 0;
    bool capped = true;   // the loop ran out of its 4096 trials
    while (trial < 4096) {
      if (trial > 0 && alam != 1.0 && xfin) {
        const double alam_b = 0.5 * alam;
        const double ha = partial_half_sum(alam);
        const double hb = partial_half_sum(alam_b);
        if (ha > sf_thr) {            // trial `trial` fails
          ++trials;
          if (alam < alamin) {
            capped = false;
            stale = true;
            break;
          }
          alam = alam_b;
          if (++trial >= 4096) break;
          if (alam != 1.0 && hb > sf_thr) {   // and so does the next one
            ++trials;
            if (alam < alamin) {
              capped = false;
              stale = true;
              break;
            }
            alam = 0.5 * alam;
            ++trial;
            continue;
          }
        }
      }
      // a trial with the full residual
      double qt[NV];
#pragma unroll
      for (int i = 0; i < NV; ++i) qj_rel[i] = x_old[i] + alam * dd[i];
#pragma unroll
      for (int i = 0; i < NV; ++i) qt[i] = qj_rel[i] * qj_org[i];
      eval_f<NS>(P, qt, qj_old, Rj, bx, by, dt, rt, scal_f);
      ++trials;
      if (scal_f <= sf_thr) {
        capped = false;
        break;
      }
      if (alam < alamin) {
        capped = false;
        stale = true;
        break;
      }
      if (alam == 1.0) {
        double tmplam = -slope / (2.0 * (scal_f - scal_f_old - slope));
        alam = fmax_f(tmplam, 0.5 * alam);
      } else {
        alam = 0.5 * alam;
      }
      ++trial;
    }
    if (stale || capped) {
      // alam < alamin or the trial cap: the old iterate is put back
#pragma unroll
      for (int i = 0; i < NV; ++i) qj_rel[i] = x_old[i];
      scal_f = scal_f_old;
      stale = true;
    }
  }
#pragma unroll
  for (int i = 0; i < NV; ++i) qj[i] = qj_rel[i] * qj_org[i];
  return newton_converged<NS>(rt, qj_rel, x_old);
}

// ============================================================ mass exchange
template <int NS>
IMEX_FLAT void mass_exchange(const DevParams& P, const double* qpj, double bx, double by,
                              const double* erod, double dtl, double* ers, double* dep,
                              double& cpe, double& cpl, double* eqns, double& topo,
                              bool& dep_neg) {
  constexpr int NV = 4 + NS;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    ers[i] = 0.0;
    dep[i] = 0.0;
  }
  cpe = 0.0;
  cpl = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) eqns[i] = 0.0;
  topo = 0.0;
  if (qpj[0] <= EPS) return;
  const double alpha_max = 0.6, hind_exp = 4.65;
  double r_h = qpj[0], r_u = qpj[NV], r_v = qpj[NV + 1];
  double al[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) al[i] = P.alpha_flag ? qpj[4 + i] : qpj[4 + i] / qpj[0];
  double at = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) at += al[i];
  double r_w = P.slope_correction_flag ? (r_u * bx + r_v * by) : 0.0;
  double mv2 = r_u * r_u + r_v * r_v + r_w * r_w;
  double mv = sqrt(mv2);
  double tse;
  if (P.erosion_coeff > 0.0) {
    double te = P.erosion_coeff * mv * r_h * (1.0 - at);
    tse = te * (1.0 - P.erodible_porosity);
#pragma unroll
    for (int i = 0; i < NS; ++i) ers[i] = P.erodible_fract[i] * tse;
  }
#pragma unroll
  for (int i = 0; i < NS; ++i) ers[i] = fmax_f(0.0, fmin_f(ers[i], erod[i] / dtl));
  tse = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) tse += ers[i];
  double te = tse / (1.0 - P.erodible_porosity);
  cpe = te * P.erodible_porosity;
  if (at <= P.alphastot_min) return;
  double r_T = qpj[3];
  Mixt m = mixt_var<NS>(P, qpj);
  double spc = sp_heat_c_of<NS>(P, qpj, m.rho_m);
  double ikv = 1.0 / P.kin_visc_c;
  double hind = -1.0;   // the hindered-settling factor, the same for every class
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    if (al[i] > 0.0 && P.settling_flag) {
      double sv = settling_velocity(P, P.diam_s[i], P.rho_s[i], m.rho_c, ikv);
      dep[i] = al[i] * sv * 1.0;
      if (hind < 0.0) hind = ipow(1.0 - fmin_f(1.0, at / alpha_max), hind_exp);
      dep[i] = dep[i] * hind;
      dep[i] = fmin_f(dep[i], r_h * al[i] / dtl);
      if (dep[i] < 0.0) dep_neg = true;
    }
  }
  double sdep = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sdep += dep[i];
  cpl = 0.0;
  cpl = cpl + P.coeff_porosity * sdep;
  double sal = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sal += al[i];
  cpl = fmin_f(cpl, r_h * fmax_f(0.0, P.maximum_solid_packing - sal) / dtl);
  cpl = fmin_f(cpl, (r_h * (1.0 - sal) - P.coeff_porosity * (r_h * sal - dtl * sdep)) / dtl);
  double T_erod = P.erodible_deposit_flag ? r_T : P.T_erodible;
  double air_entr = 0.0;
  if (P.entrainment_flag && r_h > 0.0 && m.Ri > 0.0) {
    double entr_coeff = 0.075 / sqrt(1.0 + 718.0 * ipow(m.Ri, 2.4));
    air_entr = entr_coeff * sqrt(mv2);
  }
  double dep_tot = 0.0, ers_tot = 0.0, rdt = 0.0, ret = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) dep_tot += dep[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) ers_tot += ers[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) rdt += P.rho_s[i] * dep[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) ret += P.rho_s[i] * ers[i];
  eqns[0] = P.rho_a_amb * air_entr + ret - rdt + P.rho_c_sub * cpe - m.rho_c * cpl;
  eqns[1] = -(r_u * (rdt + m.rho_c * cpl));
  eqns[2] = -(r_v * (rdt + m.rho_c * cpl));
  double sdh = 0.0, seh = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) sdh += P.rho_s[i] * P.sp_heat_s[i] * dep[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) seh += P.rho_s[i] * P.sp_heat_s[i] * ers[i];
  if (P.energy_flag)
    eqns[3] = -(r_T * (sdh + m.rho_c * spc * cpl)) - 0.5 * mv2 * (rdt + m.rho_c * cpl) +
              T_erod * (seh + P.rho_c_sub * spc * cpe) +
              P.T_ambient * P.sp_heat_a * P.rho_a_amb * air_entr;
  else
    eqns[3] = -(r_T * (sdh + m.rho_c * spc * cpl)) + T_erod * (seh + P.rho_c_sub * spc * cpe) +
              P.T_ambient * P.sp_heat_a * P.rho_a_amb * air_entr;
#pragma unroll
  for (int i = 0; i < NS; ++i) eqns[4 + i] = P.rho_s[i] * (ers[i] - dep[i]);
  topo = (dep_tot - ers_tot) / (1.0 - P.erodible_porosity);
}

// update_erosion_deposition_cell for one cell (src/solver_2d.f90:2431-2588).
template <int NS>
__device__ bool erosion_cell(const DevParams& P, double* qc, double bx, double by,
                             double* erod, double* depo, double* eros, double* Bc,
                             double dtl) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  double qpv[NP];
  cell_qp<NS>(P, qc, qpv);
  double ers[NS], dep[NS], cpe, cpl, eqns[NV], topo;
  bool bad = false;
  mass_exchange<NS>(P, qpv, bx, by, erod, dtl, ers, dep, cpe, cpl, eqns, topo, bad);
#pragma unroll
  for (int i = 0; i < NV; ++i) qc[i] = qc[i] + dtl * eqns[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) qc[4 + i] = fmax_f(0.0, qc[4 + i]);
#pragma unroll
  for (int i = 0; i < NS; ++i) depo[i] = depo[i] + dtl * dep[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) eros[i] = eros[i] + dtl * ers[i];
#pragma unroll
  for (int i = 0; i < NS; ++i) erod[i] = erod[i] - dtl * ers[i];
  if (P.erodible_deposit_flag) {
#pragma unroll
    for (int i = 0; i < NS; ++i) erod[i] = erod[i] + dtl * dep[i];
  }
  if (P.topo_change_flag) *Bc = *Bc + dtl * topo;
#pragma unroll
  for (int i = 0; i < NS; ++i) bad |= (qc[4 + i] < 0.0);
  if (qc[0] <= 0.0) {
    if (qc[0] > -1.0e-10) {
#pragma unroll
      for (int i = 0; i < NV; ++i) qc[i] = 0.0;
    } else {
      bad = true;
    }
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) s += qc[4 + i];
  if (s > qc[0]) {
    if (qc[0] < 1.0e-10) {
      double s2 = 0.0;
#pragma unroll
      for (int i = 0; i < NS; ++i) s2 += qc[4 + i];
#pragma unroll
      for (int i = 0; i < NS; ++i) qc[4 + i] = qc[4 + i] / s2 * qc[0];
    } else {
      bad = true;
    }
  }
  double red_grav = 0.0;
  if (qc[0] > 0.0) {
    qc_to_qp<NS>(P, qc, qpv);
    red_grav = mixt_var<NS>(P, qpv).red_grav;
  }
  if (red_grav <= 0.0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = 0.0;
  }
  return bad;
}

// =============================================================== stage 2
// RK stage 2 (src/solver_2d.f90:1105-1628) as passes over the solve cells:
//   k_stage2_first   q_fv, semi-implicit terms, q_si, Rj_not_impl, Newton
//                    scaling and iteration 1; cells that go on are appended
//                    to list 0
//   k_stage2_iter    one Newton iteration (nl_iter = 2 or 3) over a list;
//                    cells that go on are appended to the next list
//   k_stage2_tail    iterations 4..100 for the few cells still iterating
//   k_stage2_post    sign guard, assemble_sol checks and fixes, q written
// Between passes a cell's Newton state (qj_rel, the residual, its norm) is
// kept in the NewtonWork planes; the iterate is carried bit for bit, so a
// cell's arithmetic is that of one uninterrupted solve_rk_step.  Iteration
// counts differ from cell to cell (mostly 2 or 3 here); running each
// iteration as its own pass over the cells that need it keeps a warp's
// lanes on the same iteration.
struct NewtonWork {
  double* qsi;    // nv planes: q_si, the Newton initial guess (scaling source)
  double* Rj;     // nv planes: Rj_not_impl
  double* x;      // nv planes: qj_rel while iterating, the final qj when done
  double* rt;     // nv planes: residual
  double* sf;     // 1 plane: 0.5*|residual|^2
  uint8_t* status;  // 1 plane: bit 0 the cell went through Newton, bit 1 its
                    // residual must be evaluated again (see newton_iterk)
  uint32_t* list[3];  // cells (k*pitch + j) still iterating after pass 0, 1, 2
  // learned warm start (warm != 0): the Newton cells of the step, their
  // network inputs and the network's momentum guesses
  int warm;
  uint32_t* wlist;    // Newton cells, in append order
  uint32_t* flist;    // warm starts to redo from q_si (k_stage2_fallback)
  float* feat;        // WARM_IN floats per wlist entry
  double* guess;      // 2 planes: proposed q(2), q(3)
  // training pairs (harvest != 0): inputs and targets of every `stride`-th
  // Newton cell, up to `cap` pairs
  int harvest;
  unsigned int hstride;
  unsigned long long hcap;
  float* hx;
  float* hy;
};

// Network inputs of one Newton cell: class-count independent quantities of
// q_si, the old state, the explicit tendency, dt and the slope.  Targets:
// the change of the two momentum components over the Newton solve, per unit
// of q(1).
constexpr int WARM_IN = 12, WARM_OUT = 2;

template <int NS>
__device__ __forceinline__ void warm_features(const double* qsi, const double* q0,
                                              const double* Rj, double dt, double bx,
                                              double by, float* f) {
  const double m = qsi[0], im = 1.0 / m;
  double xs = 0.0;
#pragma unroll
  for (int i = 0; i < NS; ++i) xs += qsi[4 + i];
  f[0] = (float)log10(fmax(m, 1.0e-12));
  f[1] = (float)(qsi[1] * im);
  f[2] = (float)(qsi[2] * im);
  f[3] = (float)(q0[1] * im);
  f[4] = (float)(q0[2] * im);
  f[5] = (float)(dt * Rj[1] * im);
  f[6] = (float)(dt * Rj[2] * im);
  f[7] = (float)(qsi[3] * im * 1.0e-6);
  f[8] = (float)(xs * im);
  f[9] = (float)log10(dt);
  f[10] = (float)bx;
  f[11] = (float)by;
}

struct WarmNorm {
  float x_mean[WARM_IN], x_std[WARM_IN], y_mean[WARM_OUT], y_std[WARM_OUT];
};

constexpr int STAGE2_THREADS = 128;

__device__ __forceinline__ unsigned int list_append(bool add, uint32_t c, uint32_t* list,
                                                    unsigned int* count) {
  const unsigned m = __ballot_sync(0xffffffffu, add);
  if (!m) return 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  unsigned int base = 0;
  if (lane == leader) base = atomicAdd(count, (unsigned int)__popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  const unsigned int slot = base + __popc(m & ((1u << lane) - 1u));
  if (add) list[slot] = c;
  return add ? slot : 0xffffffffu;
}

// Newton statistics of the cells that finished in this warp iteration
// (iters = 0: no cell finished in this lane).
__device__ __forceinline__ void newton_finish_stats(DevClock* clk, int iters,
                                                    unsigned long long& it_sum,
                                                    unsigned long long& maxit) {
  const int bin = iters > 0 ? (iters < 16 ? iters - 1 : 15) : -1;
  const unsigned peers = __match_any_sync(0xffffffffu, bin);
  if (bin >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1)
    atomicAdd(&clk->hist[bin], (unsigned long long)__popc(peers));
  if (iters > 0) {
    it_sum += (unsigned long long)iters;
    if (iters >= NEWTON_MAX_IT) maxit += 1;
  }
}

__device__ __forceinline__ void newton_flush_stats(DevClock* clk, unsigned long long cells,
                                                   unsigned long long it_sum,
                                                   unsigned long long trials,
                                                   unsigned long long maxit) {
  for (int off = 16; off > 0; off >>= 1) {
    cells += __shfl_down_sync(0xffffffffu, cells, off);
    it_sum += __shfl_down_sync(0xffffffffu, it_sum, off);
    trials += __shfl_down_sync(0xffffffffu, trials, off);
    maxit += __shfl_down_sync(0xffffffffu, maxit, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (cells) atomicAdd(&clk->newton_cells, cells);
    if (it_sum) atomicAdd(&clk->newton_iters, it_sum);
    if (trials) atomicAdd(&clk->lnsrch_trials, trials);
    if (maxit) atomicAdd(&clk->newton_maxit, maxit);
  }
}

template <int NS>
__device__ __forceinline__ bool all_finite(const double* v) {
  bool ok = true;
#pragma unroll
  for (int i = 0; i < 4 + NS; ++i) ok &= isfinite(v[i]);
  return ok;
}

// Fallback of a warm start that failed (no convergence in 100 iterations, or
// a non-finite result): the plain solve_rk_step from q_si.  Returns its
// iteration count; qj receives its result.  Run by k_stage2_fallback only.
template <int NS>
__device__ __forceinline__ int newton_plain(const DevParams& P, const NewtonWork& W, size_t c,
                                         const double* q0, const double* Rj, double bx,
                                         double by, double dt, double* qj,
                                         unsigned long long& trials) {
  constexpr int NV = 4 + NS;
  const size_t N = (size_t)P.plane;
  double qj_org[NV], qj_rel[NV], rt[NV], scal_f;
#pragma unroll
  for (int i = 0; i < NV; ++i) qj[i] = W.qsi[c + i * N];
  newton_scale<NS>(qj, qj_org);
  if (newton_start<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f)) return 1;
  if (newton_iter1<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f)) return 1;
  bool stale = false;
  int it;
  for (it = 2; it <= NEWTON_MAX_IT; ++it) {
    long long tr = 0;
    bool done = newton_iterk<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f, tr, stale);
    trials += (unsigned long long)tr;
    if (done) break;
  }
  return it > NEWTON_MAX_IT ? NEWTON_MAX_IT : it;
}

// Stage 2 up to Newton iteration 1 for one lane's cell (plane index c; the
// lane takes part in the warp's list appends whether or not it has a cell).
template <int NS>
__device__ __forceinline__ void stage2_first_lane(
    const DevParams& P, const double* __restrict__ q, const double* __restrict__ X,
    const uint8_t* __restrict__ mask, const double* __restrict__ Bx,
    const double* __restrict__ By, const double* __restrict__ Bxx,
    const double* __restrict__ Bxy, const double* __restrict__ Byy,
    const double* __restrict__ gc, NewtonWork W, DevClock* clk, double dt, bool valid,
    size_t c, unsigned long long& cells, unsigned long long& it_sum,
    unsigned long long& maxit) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const size_t N = (size_t)P.plane;
  bool go_on = false, warm_cell = false;
  int fin = 0;
  float fw[WARM_IN];
  if (valid) {
      if (mask[c]) {
        double q0[NV], qfv[NV], Xc[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
          q0[i] = q[c + i * N];
          Xc[i] = X[c + i * N];
        }
        // q_fv = q0 - dt*(MATMUL(divFlux-expl, a_tilde) - MATMUL(NH+SI_NH, a_dirk))
#pragma unroll
        for (int i = 0; i < NV; ++i) {
          double sa = (0.0 + Xc[i] * 1.0) + (0.0 - 0.0) * 0.0;
          double sb = (0.0 + (0.0 + 0.0) * 0.0) + (0.0 + 0.0) * 0.0;
          qfv[i] = q0[i] - dt * (sa - sb);
        }
        double qg[NV];
        if (qfv[0] > 0.0) {
          double qpv[NP];
          qc_to_qp<NS>(P, qfv, qpv);
          const double bx = Bx[c], by = By[c];
          double bxx = 0.0, bxy = 0.0, byy = 0.0, gcf = 1.0;
          if (P.curvature_term_flag) {
            bxx = Bxx[c];
            bxy = Bxy[c];
            byy = Byy[c];
          }
          if (P.slope_correction_flag) gcf = gc[c];
          double si2, si3;
          semi_impl_terms<NS>(P, bx, by, bxx, bxy, byy, gcf, qpv, si2, si3);
          double SI[NV], qsi[NV];
#pragma unroll
          for (int i = 0; i < NV; ++i) SI[i] = (i == 1) ? si2 : ((i == 2) ? si3 : 0.0);
#pragma unroll
          for (int i = 0; i < NV; ++i) qsi[i] = qfv[i] + dt * 1.0 * SI[i];
          if (qfv[1] * qfv[1] + qfv[2] * qfv[2] == 0.0) {
            qsi[1] = 0.0;
            qsi[2] = 0.0;
          } else if (qsi[1] * qfv[1] < 0.0 || qsi[2] * qfv[2] < 0.0) {
            qsi[1] = 0.0;
            qsi[2] = 0.0;
          } else {
            double Sm = sqrt(qsi[1] * qsi[1] + qsi[2] * qsi[2]);
            double Fm = sqrt(qfv[1] * qfv[1] + qfv[2] * qfv[2]);
            qsi[1] = Sm * qfv[1] / Fm;
            qsi[2] = Sm * qfv[2] / Fm;
          }
          double Rj[NV];
#pragma unroll
          for (int i = 0; i < NV; ++i) {
            // rows other than 2, 3: qsi = qfv + dt*0 (or +0 for qfv = -0), so
            // for finite qfv and a finite dt > 0 the difference is +0 and so
            // is the quotient
            if (i != 1 && i != 2 && isfinite(qfv[i]) && dt > 0.0 && dt < 1e300) SI[i] = 0.0;
            else SI[i] = (qsi[i] - qfv[i]) / (dt * 1.0);
            double sa = 0.0 + Xc[i] * 1.0;
            double sb = 0.0 + (0.0 + 0.0) * 0.0;
            Rj[i] = (sa - sb) - 1.0 * SI[i];
            qg[i] = qsi[i];
            W.qsi[c + i * N] = qsi[i];
            W.Rj[c + i * N] = Rj[i];
          }
          W.status[c] = 1;
          cells += 1;
          double qj_org[NV], qj_rel[NV], rt[NV], scal_f;
          if (W.warm) {
            // Newton waits for the network's guess (k_warm_predict, k_stage2_wstart)
            warm_features<NS>(qsi, q0, Rj, dt, bx, by, fw);
            warm_cell = true;
          } else {
          newton_scale<NS>(qg, qj_org);
          if (newton_start<NS>(P, qg, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f)) {
            fin = 1;
          } else if (newton_iter1<NS>(P, qg, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f)) {
            fin = 1;
          } else {
            go_on = true;
#pragma unroll
            for (int i = 0; i < NV; ++i) {
              W.x[c + i * N] = qj_rel[i];
              W.rt[c + i * N] = rt[i];
            }
            W.sf[c] = scal_f;
          }
          }
        } else {
#pragma unroll
          for (int i = 0; i < NV; ++i) qg[i] = qfv[i];
          W.status[c] = 0;
        }
        if (!go_on && !warm_cell) {
#pragma unroll
          for (int i = 0; i < NV; ++i) W.x[c + i * N] = qg[i];
        }
      }
    }
  newton_finish_stats(clk, fin, it_sum, maxit);
  list_append(go_on, (uint32_t)c, W.list[0], &clk->nw_count[0]);
  if (W.warm) {
    const unsigned int slot = list_append(warm_cell, (uint32_t)c, W.wlist, &clk->nw_count[3]);
    if (warm_cell) {
#pragma unroll
      for (int i = 0; i < WARM_IN; ++i) W.feat[(size_t)slot * WARM_IN + i] = fw[i];
    }
  }
}

// k_stage2_first: 80 registers (6 blocks of 128 per SM) measured faster
// than 64 with its larger spill set.
#ifndef IMEX_FIRST_MINB
#define IMEX_FIRST_MINB 6
#endif
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_FIRST_MINB)
    k_stage2_first(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                   const double* __restrict__ X, const uint8_t* __restrict__ mask,
                   const double* __restrict__ Bx, const double* __restrict__ By,
                   const double* __restrict__ Bxx, const double* __restrict__ Bxy,
                   const double* __restrict__ Byy, const double* __restrict__ gc, NewtonWork W,
                   DevClock* clk) {
  const DevParams& P = Pp;
  const int nx = P.nx;
  const long long ncell = (long long)nx * P.ny;
  const double dt = clk->dt;
  unsigned long long cells = 0, it_sum = 0, maxit = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < ncell;
       base += stride) {
    const long long g = base + (threadIdx.x & 31);
    const bool valid = g < ncell;
    const size_t c = valid ? (size_t)(g / nx) * P.pitch + (size_t)(g % nx) : 0;
    stage2_first_lane<NS>(P, q, X, mask, Bx, By, Bxx, Bxy, Byy, gc, W, clk, dt, valid, c, cells,
                          it_sum, maxit);
  }
  newton_flush_stats(clk, cells, it_sum, 0, maxit);
}

// One Newton iteration (nl_iter = 2 or 3) for entry e of list nl_iter-2
// (valid: e is inside the list); the lane takes part in the warp's list
// appends whether or not it has a cell.
template <int NS>
__device__ __forceinline__ void stage2_iter_lane(const DevParams& P, const double* __restrict__ q,
                                                 const double* __restrict__ Bx,
                                                 const double* __restrict__ By, NewtonWork W,
                                                 DevClock* clk, double dt, int nl_iter,
                                                 bool valid, long long e,
                                                 unsigned long long& it_sum,
                                                 unsigned long long& maxit,
                                                 unsigned long long& trials) {
  constexpr int NV = 4 + NS;
  const size_t N = (size_t)P.plane;
  const uint32_t* in = W.list[nl_iter - 2];
  uint32_t* out = W.list[nl_iter - 1];
  {
    uint32_t c = 0;
    bool go_on = false, fb = false;
    int fin = 0;
    if (valid) {
      c = in[e];
      double q0[NV], Rj[NV], qj_org[NV], qj_rel[NV], rt[NV], qj[NV], scal_f;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        q0[i] = q[c + i * N];
        Rj[i] = W.Rj[c + i * N];
        qj[i] = W.qsi[c + i * N];
        qj_rel[i] = W.x[c + i * N];
        rt[i] = W.rt[c + i * N];
      }
      if (W.warm) {   // the Newton start (scaling source) was the network's guess
        qj[1] = W.guess[c];
        qj[2] = W.guess[c + N];
      }
      scal_f = W.sf[c];
      bool stale = (W.status[c] & 2) != 0;
      newton_scale<NS>(qj, qj_org);
      long long tr = 0;
      bool done = newton_iterk<NS>(P, qj, q0, Rj, Bx[c], By[c], dt, qj_org, qj_rel, rt, scal_f, tr,
                                   stale);
      trials += (unsigned long long)tr;
      if (done || nl_iter >= NEWTON_MAX_IT) {
        fin = nl_iter;
        if (W.warm && (!done || !all_finite<NS>(qj))) {
          fb = true;
        } else {
#pragma unroll
          for (int i = 0; i < NV; ++i) W.x[c + i * N] = qj[i];
        }
      } else {
        go_on = true;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
          W.x[c + i * N] = qj_rel[i];
          W.rt[c + i * N] = rt[i];
        }
        W.sf[c] = scal_f;
        W.status[c] = stale ? 3 : 1;
      }
    }
    newton_finish_stats(clk, fin, it_sum, maxit);
    list_append(go_on, c, out, &clk->nw_count[nl_iter - 1]);
    if (W.warm) list_append(fb, c, W.flist, &clk->nw_fb);
  }
}

template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    k_stage2_iter(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                  const double* __restrict__ Bx, const double* __restrict__ By, NewtonWork W,
                  DevClock* clk, int nl_iter) {
  const DevParams& P = Pp;
  const double dt = clk->dt;
  const long long n = (long long)clk->nw_count[nl_iter - 2];
  unsigned long long it_sum = 0, maxit = 0, trials = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long e = base + (threadIdx.x & 31);
    stage2_iter_lane<NS>(P, q, Bx, By, W, clk, dt, nl_iter, e < n, e, it_sum, maxit, trials);
  }
  newton_flush_stats(clk, 0, it_sum, trials, maxit);
}

// Iterations 4..100 for entry e of list 2.
template <int NS>
__device__ __forceinline__ void stage2_tail_lane(const DevParams& P, const double* __restrict__ q,
                                                 const double* __restrict__ Bx,
                                                 const double* __restrict__ By, NewtonWork W,
                                                 DevClock* clk, double dt, bool valid,
                                                 long long e, unsigned long long& it_sum,
                                                 unsigned long long& maxit,
                                                 unsigned long long& trials) {
  constexpr int NV = 4 + NS;
  const size_t N = (size_t)P.plane;
  {
    int fin = 0;
    bool fb = false;
    uint32_t c = 0;
    if (valid) {
      c = W.list[2][e];
      double q0[NV], Rj[NV], qj_org[NV], qj_rel[NV], rt[NV], qj[NV], scal_f;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        q0[i] = q[c + i * N];
        Rj[i] = W.Rj[c + i * N];
        qj[i] = W.qsi[c + i * N];
        qj_rel[i] = W.x[c + i * N];
        rt[i] = W.rt[c + i * N];
      }
      if (W.warm) {
        qj[1] = W.guess[c];
        qj[2] = W.guess[c + N];
      }
      scal_f = W.sf[c];
      bool stale = (W.status[c] & 2) != 0;
      newton_scale<NS>(qj, qj_org);
      const double bx = Bx[c], by = By[c];
      int it;
      for (it = 4; it <= NEWTON_MAX_IT; ++it) {
        long long tr = 0;
        bool done = newton_iterk<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f, tr,
                                     stale);
        trials += (unsigned long long)tr;
        if (done) break;
      }
      fin = it > NEWTON_MAX_IT ? NEWTON_MAX_IT : it;
      if (W.warm && (it > NEWTON_MAX_IT || !all_finite<NS>(qj))) {
        fb = true;
      } else {
#pragma unroll
        for (int i = 0; i < NV; ++i) W.x[c + i * N] = qj[i];
      }
    }
    newton_finish_stats(clk, fin, it_sum, maxit);
    if (W.warm) list_append(fb, c, W.flist, &clk->nw_fb);
  }
}

template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    k_stage2_tail(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                  const double* __restrict__ Bx, const double* __restrict__ By, NewtonWork W,
                  DevClock* clk) {
  const DevParams& P = Pp;
  const double dt = clk->dt;
  const long long n = (long long)clk->nw_count[2];
  unsigned long long it_sum = 0, maxit = 0, trials = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long e = base + (threadIdx.x & 31);
    stage2_tail_lane<NS>(P, q, Bx, By, W, clk, dt, e < n, e, it_sum, maxit, trials);
  }
  newton_flush_stats(clk, 0, it_sum, trials, maxit);
}

// The network's momentum guesses for the cells of the warm-start list:
// 16 cells per warp through the tensor-core forward pass.
template <int NS>
__global__ void __launch_bounds__(32 * mlp::WARPS)
    k_warm_predict(const __grid_constant__ DevParams Pp, NewtonWork W, DevClock* clk,
                   const __nv_bfloat16* __restrict__ gW, const float* __restrict__ gP,
                   WarmNorm nrm) {
  const DevParams& P = Pp;
  const size_t N = (size_t)P.plane;
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
  float* sP = reinterpret_cast<float*>(smem + mlp::NBW * sizeof(__nv_bfloat16));
  __shared__ float xin[mlp::WARPS][16 * WARM_IN];
  __shared__ float yout[mlp::WARPS][16 * WARM_OUT];
  mlp::load_net(gW, gP, sW, sP);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long n = (long long)clk->nw_count[3];
  for (long long r0 = ((long long)blockIdx.x * mlp::WARPS + warp) * 16; r0 < n;
       r0 += (long long)gridDim.x * mlp::WARPS * 16) {
    const int nv = (int)((n - r0) < 16 ? (n - r0) : 16);
    for (int e = lane; e < 16 * WARM_IN; e += 32) {
      const int r = e / WARM_IN, k = e % WARM_IN;
      xin[warp][e] = r < nv ? (W.feat[(size_t)(r0 + r) * WARM_IN + k] - nrm.x_mean[k]) / nrm.x_std[k]
                            : 0.0f;
    }
    __syncwarp();
    mlp::forward16(xin[warp], nv, sW, sP, yout[warp], WARM_OUT, nullptr);
    __syncwarp();
    if (lane < nv) {
      const uint32_t c = W.wlist[r0 + lane];
      const double m = W.qsi[c];
#pragma unroll
      for (int k = 0; k < WARM_OUT; ++k) {
        const double tk = (double)yout[warp][lane * WARM_OUT + k] * nrm.y_std[k] + nrm.y_mean[k];
        W.guess[c + k * N] = W.qsi[c + (1 + k) * N] + m * tk;
      }
    }
    __syncwarp();
  }
}

// Newton scaling and iteration 1 from the network's guess for the cells of
// the warm-start list; cells still iterating go to list 0 as in
// k_stage2_first.
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    k_stage2_wstart(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                    const double* __restrict__ Bx, const double* __restrict__ By, NewtonWork W,
                    DevClock* clk) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS;
  const size_t N = (size_t)P.plane;
  const double dt = clk->dt;
  const long long n = (long long)clk->nw_count[3];
  unsigned long long it_sum = 0, maxit = 0, trials = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < n;
       base += stride) {
    const long long e = base + (threadIdx.x & 31);
    uint32_t c = 0;
    bool go_on = false, fb = false;
    int fin = 0;
    if (e < n) {
      c = W.wlist[e];
      double q0[NV], Rj[NV], qj[NV], qj_org[NV], qj_rel[NV], rt[NV], scal_f;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        q0[i] = q[c + i * N];
        Rj[i] = W.Rj[c + i * N];
        qj[i] = W.qsi[c + i * N];
      }
      qj[1] = W.guess[c];
      qj[2] = W.guess[c + N];
      const double bx = Bx[c], by = By[c];
      newton_scale<NS>(qj, qj_org);
      bool done = newton_start<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f) ||
                  newton_iter1<NS>(P, qj, q0, Rj, bx, by, dt, qj_org, qj_rel, rt, scal_f);
      if (done) {
        fin = 1;
        if (!all_finite<NS>(qj)) {
          fb = true;
        } else {
#pragma unroll
          for (int i = 0; i < NV; ++i) W.x[c + i * N] = qj[i];
        }
      } else {
        go_on = true;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
          W.x[c + i * N] = qj_rel[i];
          W.rt[c + i * N] = rt[i];
        }
        W.sf[c] = scal_f;
      }
    }
    newton_finish_stats(clk, fin, it_sum, maxit);
    list_append(go_on, c, W.list[0], &clk->nw_count[0]);
    list_append(fb, c, W.flist, &clk->nw_fb);
  }
  newton_flush_stats(clk, 0, it_sum, trials, maxit);
}

// Warm starts that failed, redone with the plain start (q_si).
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS, IMEX_STAGE2_MINB)
    k_stage2_fallback(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                      const double* __restrict__ Bx, const double* __restrict__ By,
                      NewtonWork W, DevClock* clk) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS;
  const size_t N = (size_t)P.plane;
  const double dt = clk->dt;
  const long long n = (long long)clk->nw_fb;
  unsigned long long it_sum = 0, trials = 0;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const uint32_t c = W.flist[e];
    double q0[NV], Rj[NV], qj[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      q0[i] = q[c + i * N];
      Rj[i] = W.Rj[c + i * N];
    }
    it_sum += (unsigned long long)newton_plain<NS>(P, W, c, q0, Rj, Bx[c], By[c], dt, qj, trials);
#pragma unroll
    for (int i = 0; i < NV; ++i) W.x[c + i * N] = qj[i];
    atomicAdd(&clk->warm_fallback, 1ULL);
  }
  if (it_sum) atomicAdd(&clk->newton_iters, it_sum);
  if (trials) atomicAdd(&clk->lnsrch_trials, trials);
}

// Training pairs from the finished Newton solves (before the sign guard):
// the inputs of warm_features and the momentum change per unit q(1), for
// every hstride-th Newton cell (cells taken by a hash of their index and
// the step, so that successive steps sample different cells).
template <int NS>
__global__ void __launch_bounds__(128)
    k_harvest(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
              const double* __restrict__ Bx, const double* __restrict__ By, NewtonWork W,
              DevClock* clk) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS;
  const int nx = P.nx;
  const long long ncell = (long long)nx * P.ny;
  const size_t N = (size_t)P.plane;
  const double dt = clk->dt;
  const unsigned long long salt = clk->steps * 0x9E3779B97F4A7C15ULL;
  for (long long base = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < ncell;
       base += (long long)gridDim.x * blockDim.x) {
    const long long g = base + (threadIdx.x & 31);
    bool take = false;
    size_t c = 0;
    float f[WARM_IN], y[WARM_OUT];
    if (g < ncell) {
      c = (size_t)(g / nx) * P.pitch + (size_t)(g % nx);
      unsigned long long h = ((unsigned long long)g + salt) * 0xBF58476D1CE4E5B9ULL;
      h ^= h >> 31;
      if ((W.status[c] & 1) && (h % W.hstride) == 0) {
        double q0[NV], qsi[NV], Rj[NV], x1, x2;
#pragma unroll
        for (int i = 0; i < NV; ++i) {
          q0[i] = q[c + i * N];
          qsi[i] = W.qsi[c + i * N];
          Rj[i] = W.Rj[c + i * N];
        }
        x1 = W.x[c + N];
        x2 = W.x[c + 2 * N];
        if (qsi[0] > 0.0 && isfinite(x1) && isfinite(x2)) {
          warm_features<NS>(qsi, q0, Rj, dt, Bx[c], By[c], f);
          y[0] = (float)((x1 - qsi[1]) / qsi[0]);
          y[1] = (float)((x2 - qsi[2]) / qsi[0]);
          take = true;
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (!m) continue;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long slot0 = 0;
    if (lane == leader) slot0 = atomicAdd(&clk->harvest_n, (unsigned long long)__popc(m));
    slot0 = __shfl_sync(0xffffffffu, slot0, leader);
    const unsigned long long slot = slot0 + __popc(m & ((1u << lane) - 1u));
    if (take && slot < W.hcap) {
#pragma unroll
      for (int i = 0; i < WARM_IN; ++i) W.hx[slot * WARM_IN + i] = f[i];
      W.hy[slot * WARM_OUT + 0] = y[0];
      W.hy[slot * WARM_OUT + 1] = y[1];
    }
  }
}

// Sign guard after Newton (src/solver_2d.f90:1238-1255) and assemble_sol
// (src/solver_2d.f90:1339-1626).
template <int NS>
__device__ __forceinline__ void stage2_post_cell(const DevParams& P, double* __restrict__ q,
                                                 const uint8_t* __restrict__ cellinfo,
                                                 NewtonWork W, DevClock* clk, int j, int k) {
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const int nx = P.nx, ny = P.ny;
  const size_t N = (size_t)P.plane;
  const size_t c = (size_t)k * P.pitch + j;
  {
    double qc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = W.x[c + i * N];
    if (W.status[c] & 1) {
      const double qs1 = W.qsi[c + N], qs2 = W.qsi[c + 2 * N];
      if (ny == 1) qc[2] = 0.0;
      if (nx == 1) qc[1] = 0.0;
      if (qs1 * qs1 + qs2 * qs2 == 0.0) {
        qc[1] = 0.0;
        qc[2] = 0.0;
      } else if (qc[1] * qs1 <= 0.0 && qc[2] * qs2 <= 0.0) {
        qc[1] = 0.0;
        qc[2] = 0.0;
      } else {
        double Sm = sqrt(qc[1] * qc[1] + qc[2] * qc[2]);
        double Fm = sqrt(qs1 * qs1 + qs2 * qs2);
        qc[1] = Sm * qs1 / Fm;
        qc[2] = Sm * qs2 / Fm;
      }
    }
    const long long cell = (long long)k * nx + j;
    bool anynan = false;
#pragma unroll
    for (int i = 0; i < NV; ++i) anynan |= isnan(qc[i]);
    if (anynan) record_error(clk, 1, cell);
    if (qc[0] < EPS) {
      if (qc[0] > -1.0e-7) {
#pragma unroll
        for (int i = 0; i < NV; ++i) qc[i] = 0.0;
      } else {
        record_error(clk, 2, cell);
      }
    }
    bool anyneg = false, anybad = false;
#pragma unroll
    for (int i = 0; i < NS; ++i) anyneg |= (qc[4 + i] < 0.0);
    if (anyneg) {
#pragma unroll
      for (int i = 0; i < NS; ++i) anybad |= (qc[4 + i] <= -1.0e-7);
      if (anybad) {
        record_error(clk, 3, cell);
      } else {
#pragma unroll
        for (int i = 0; i < NS; ++i)
          if (qc[4 + i] > -1.0e-7) qc[4 + i] = 0.0;
      }
    }
    double qpv[NP];
    qc_to_qp<NS>(P, qc, qpv);
    if (qpv[3] < 273.0) record_error(clk, 4, cell);
    double ssum = 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) ssum += qc[4 + i];
    if (ssum > qc[0]) {
      if ((ssum - qc[0]) / qc[0] < 1.0e-10 || qc[0] < EPS) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NS; ++i) s += qc[4 + i];
#pragma unroll
        for (int i = 0; i < NS; ++i) qc[4 + i] = qc[4 + i] / s * qc[0];
      } else {
        record_error(clk, 5, cell);
      }
    }
    if (P.has_cellinfo && (cellinfo[cell] & CI_NODATA)) {
#pragma unroll
      for (int i = 0; i < NV; ++i) qc[i] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < NV; ++i) q[c + i * N] = qc[i];
  }
}

template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS)
    k_stage2_post(const __grid_constant__ DevParams Pp, double* __restrict__ q,
                  const uint8_t* __restrict__ mask, const uint8_t* __restrict__ cellinfo,
                  NewtonWork W, DevClock* clk) {
  const DevParams& P = Pp;
  const int nx = P.nx;
  const long long ncell = (long long)nx * P.ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % nx), k = (int)(g / nx);
    if (!mask[(size_t)k * P.pitch + j]) continue;
    stage2_post_cell<NS>(P, q, cellinfo, W, clk, j, k);
  }
}

// k_stage2_post over the grid rows [k0, k1) (imex_gpu_advance_host).
template <int NS>
__global__ void __launch_bounds__(STAGE2_THREADS)
    k_stage2_post_rows(const __grid_constant__ DevParams Pp, double* __restrict__ q,
                       const uint8_t* __restrict__ mask, const uint8_t* __restrict__ cellinfo,
                       NewtonWork W, DevClock* clk, int k0, int k1) {
  const DevParams& P = Pp;
  const int nx = P.nx;
  const long long ncell = (long long)nx * (k1 - k0);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % nx), k = k0 + (int)(g / nx);
    if (!mask[(size_t)k * P.pitch + j]) continue;
    stage2_post_cell<NS>(P, q, cellinfo, W, clk, j, k);
  }
}

// Stand-alone erosion/deposition pass (imex_gpu_erosion_deposition).
template <int NS>
__device__ __forceinline__ void erosion_update_cell(const DevParams& P, double* __restrict__ q,
                                                    const double* __restrict__ Bx,
                                                    const double* __restrict__ By,
                                                    double* __restrict__ erodible,
                                                    double* __restrict__ deposit,
                                                    double* __restrict__ erosion,
                                                    double* __restrict__ Bcent, DevClock* clk,
                                                    double dt, int j, int k) {
  constexpr int NV = 4 + NS;
  const int nx = P.nx;
  const size_t c = (size_t)k * P.pitch + j;
  {
    double qc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = q[c + (size_t)i * P.plane];
    double er[NS], de[NS], eo[NS], Bc = 0.0;
    const size_t N = (size_t)P.plane;
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      er[i] = erodible[c + i * N];
      de[i] = deposit[c + i * N];
      eo[i] = erosion[c + i * N];
    }
    if (P.topo_change_flag) Bc = Bcent[c];
    bool bad = erosion_cell<NS>(P, qc, Bx[c], By[c], er, de, eo, &Bc, dt);
#pragma unroll
    for (int i = 0; i < NS; ++i) {
      erodible[c + i * N] = er[i];
      deposit[c + i * N] = de[i];
      erosion[c + i * N] = eo[i];
    }
    if (P.topo_change_flag) Bcent[c] = Bc;
    if (bad) record_error(clk, 6, (long long)k * nx + j);
#pragma unroll
    for (int i = 0; i < NV; ++i) q[c + (size_t)i * P.plane] = qc[i];
  }
}

template <int NS>
__global__ void __launch_bounds__(128, IMEX_EROSION_MINB)
    k_erosion(const __grid_constant__ DevParams Pp, double* __restrict__ q, const uint8_t* __restrict__ mask,
              const double* __restrict__ Bx, const double* __restrict__ By,
              double* __restrict__ erodible, double* __restrict__ deposit,
              double* __restrict__ erosion, double* __restrict__ Bcent, DevClock* clk) {
  const DevParams& P = Pp;
  const int nx = P.nx;
  const long long ncell = (long long)nx * P.ny;
  const double dt = clk->dt;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    int j = (int)(g % nx), k = (int)(g / nx);
    if (!mask[(size_t)k * P.pitch + j]) continue;
    erosion_update_cell<NS>(P, q, Bx, By, erodible, deposit, erosion, Bcent, clk, dt, j, k);
  }
}

// k_erosion over the grid rows [k0, k1) (imex_gpu_advance_host).
template <int NS>
__global__ void __launch_bounds__(128, IMEX_EROSION_MINB)
    k_erosion_rows(const __grid_constant__ DevParams Pp, double* __restrict__ q,
                   const uint8_t* __restrict__ mask, const double* __restrict__ Bx,
                   const double* __restrict__ By, double* __restrict__ erodible,
                   double* __restrict__ deposit, double* __restrict__ erosion,
                   double* __restrict__ Bcent, DevClock* clk, int k0, int k1) {
  const DevParams& P = Pp;
  const int nx = P.nx;
  const long long ncell = (long long)nx * (k1 - k0);
  const double dt = clk->dt;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % nx), k = k0 + (int)(g / nx);
    if (!mask[(size_t)k * P.pitch + j]) continue;
    erosion_update_cell<NS>(P, q, Bx, By, erodible, deposit, erosion, Bcent, clk, dt, j, k);
  }
}

// ============================================================ small kernels
// FMA-chain throughput probe: each thread runs 8 independent chains of
// `iters` dependent fused multiply-adds (the measured FP64 peak).
__global__ void k_fp64_probe(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1.0, x2 = x0 + 2.0, x3 = x0 + 3.0;
  double x4 = x0 + 4.0, x5 = x0 + 5.0, x6 = x0 + 6.0, x7 = x0 + 7.0;
  for (int i = 0; i < iters; ++i) {
    x0 = __fma_rn(x0, a, b); x1 = __fma_rn(x1, a, b); x2 = __fma_rn(x2, a, b); x3 = __fma_rn(x3, a, b);
    x4 = __fma_rn(x4, a, b); x5 = __fma_rn(x5, a, b); x6 = __fma_rn(x6, a, b); x7 = __fma_rn(x7, a, b);
  }
  double r = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (r == 12345.678) out[0] = r;  // keeps the chains live
}

// Resets the per-step accumulators of the clock.
__device__ __forceinline__ void step_begin(DevClock* clk, double max_dt, int reset_cells) {
  clk->dtmin_bits = (unsigned long long)__double_as_longlong(max_dt);
  if (reset_cells) clk->solve_cells = 0;
  clk->newton_cells = 0;
  clk->newton_iters = 0;
  clk->lnsrch_trials = 0;
  clk->newton_maxit = 0;
  clk->warm_fallback = 0;
  for (int b = 0; b < 16; ++b) clk->hist[b] = 0;
}

__global__ void k_step_begin(DevClock* clk, double max_dt, int reset_cells) {
  step_begin(clk, max_dt, reset_cells);
}

// Empties the stage-2 Newton lists (before each stage 2).
__device__ __forceinline__ void nw_reset(DevClock* clk) {
  for (int i = 0; i < 4; ++i) clk->nw_count[i] = 0;
  clk->nw_fb = 0;
}
__global__ void k_nw_reset(DevClock* clk) { nw_reset(clk); }

// dt from the CFL minimum with the driver's clipping (src/IMEX_SfloW2D.f90:359-381).
__device__ __forceinline__ void dt_clip(DevClock* clk, int clip) {
  double dt = __longlong_as_double((long long)clk->dtmin_bits);
  if (clip) {
    double t = clk->t;
    if (t + dt > clk->t_end) dt = clk->t_end - t;
    if (clk->t_output >= 0.0 && t + dt > clk->t_output) dt = clk->t_output - t;
    dt = fmin_f(dt, 1.1 * 0.5 * (clk->dt_old + clk->dt_old_old));
    clk->dt_old_old = clk->dt_old;
    clk->dt_old = dt;
  }
  clk->dt = dt;
}
__global__ void k_dt_clip(DevClock* clk, int clip) { dt_clip(clk, clip); }

__device__ __forceinline__ void step_end(DevClock* clk) {
  clk->t = clk->t + clk->dt;
  clk->steps += 1;
}
__global__ void k_step_end(DevClock* clk) { step_end(clk); }

// Fortran AoS q(n_vars,nx,ny) <-> SoA planes.
__global__ void k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int nv,
                             int nx, int ny, long long pitch, long long plane) {
  long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * nv;
       g += (long long)gridDim.x * blockDim.x) {
    long long cell = g / nv;
    int v = (int)(g % nv);
    int j = (int)(cell % nx), k = (int)(cell / nx);
    soa[(size_t)v * plane + (size_t)k * pitch + j] = aos[g];
  }
}
__global__ void k_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int nv,
                             int nx, int ny, long long pitch, long long plane) {
  long long n = (long long)nx * ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n * nv;
       g += (long long)gridDim.x * blockDim.x) {
    long long cell = g / nv;
    int v = (int)(g % nv);
    int j = (int)(cell % nx), k = (int)(cell / nx);
    aos[g] = soa[(size_t)v * plane + (size_t)k * pitch + j];
  }
}

// qp planes for imex_gpu_get_state (driver's post-step convention).
template <int NS>
__global__ void k_qp_out(const __grid_constant__ DevParams Pp, const double* __restrict__ q, double* __restrict__ qp_aos,
                         const uint8_t* __restrict__ cellinfo) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS, NP = 6 + NS;
  long long n = (long long)P.nx * P.ny;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    int j = (int)(g % P.nx), k = (int)(g / P.nx);
    size_t c = (size_t)k * P.pitch + j;
    double qc[NV], qpv[NP];
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = q[c + (size_t)i * P.plane];
    cell_qp<NS>(P, qc, qpv);
#pragma unroll
    for (int i = 0; i < NP; ++i) qp_aos[(size_t)g * NP + i] = qpv[i];
  }
}

// ==================================================== topography update
// topography_reconstruction after a bed change (src/geometry_2d.f90:683-860):
// the 5-point first and second derivatives of B_cent and the 25-point mixed
// one on the cells 3..n-2, copied to the 2-cell border; with slope
// correction, grav_coeff, its x derivative and its staggered values.  A cell
// in the border takes the stencil of its nearest interior cell, which is
// what the reference's copies leave there.
__global__ void __launch_bounds__(256)
    k_topo_geom(const __grid_constant__ DevParams Pp, const double* __restrict__ B,
                double* __restrict__ Bx, double* __restrict__ By, double* __restrict__ Bxx,
                double* __restrict__ Bxy, double* __restrict__ Byy) {
  const DevParams& P = Pp;
  const int nx = P.nx, ny = P.ny;
  const long long n = (long long)nx * ny;
  const double c1[5] = {-2.0, -1.0, 0.0, 1.0, 2.0};
  const double c2[5] = {2.0, -1.0, -2.0, -1.0, 2.0};
  const double n1x = 10.0 * P.dx, n1y = 10.0 * P.dy;
  const double n2x = 7.0 * (P.dx * P.dx), n2y = 7.0 * (P.dy * P.dy);
  const double nxy = (10.0 * P.dx) * (10.0 * P.dy);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < n;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % nx), k = (int)(g / nx);
    const int js = min(max(j, 2), nx - 3), ks = min(max(k, 2), ny - 3);
    auto b = [&](int jj, int kk) { return B[(size_t)kk * P.pitch + jj]; };
    double px = 0.0, sxx = 0.0, py = 0.0, syy = 0.0;
#pragma unroll
    for (int t = 0; t < 5; ++t) {
      px = px + c1[t] * b(js + t - 2, ks);
      sxx = sxx + c2[t] * b(js + t - 2, ks);
    }
#pragma unroll
    for (int t = 0; t < 5; ++t) {
      py = py + c1[t] * b(js, ks + t - 2);
      syy = syy + c2[t] * b(js, ks + t - 2);
    }
    double ws = 0.0;
    for (int u = 0; u < 5; ++u)
#pragma unroll
      for (int t = 0; t < 5; ++t) ws = ws + c1[t] * c1[u] * b(js + t - 2, ks + u - 2);
    const size_t c = (size_t)k * P.pitch + j;
    Bx[c] = px / n1x;
    By[c] = py / n1y;
    if (Bxx) {
      Bxx[c] = sxx / n2x;
      Byy[c] = syy / n2y;
      Bxy[c] = ws / nxy;
    }
  }
}

__device__ __forceinline__ double topo_gc(double bx, double by) {
  return 1.0 / (1.0 + bx * bx + by * by);
}

__global__ void __launch_bounds__(256)
    k_topo_gc(const __grid_constant__ DevParams Pp, const double* __restrict__ Bx,
              const double* __restrict__ By, const double* __restrict__ Bxx,
              const double* __restrict__ Bxy, double* __restrict__ gc, double* __restrict__ dgc,
              double* __restrict__ gcsx, double* __restrict__ gcsy) {
  const DevParams& P = Pp;
  const int nx = P.nx, ny = P.ny;
  const long long ncell = (long long)nx * ny, nsx = (long long)(nx + 1) * ny,
                  nsy = (long long)nx * (ny + 1);
  auto gcat = [&](int j, int k) {
    const size_t c = (size_t)k * P.pitch + j;
    return topo_gc(Bx[c], By[c]);
  };
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell + nsx + nsy;
       g += (long long)gridDim.x * blockDim.x) {
    if (g < ncell) {
      const int j = (int)(g % nx), k = (int)(g / nx);
      const size_t c = (size_t)k * P.pitch + j;
      const double bx = Bx[c], by = By[c], gcv = topo_gc(bx, by);
      gc[c] = gcv;
      dgc[c] = -(2.0 * (gcv * gcv) * (bx * Bxx[c] + by * Bxy[c]));
    } else if (g < ncell + nsx) {
      const long long h = g - ncell;           // grav_coeff_stag_x(nx+1, ny)
      const int j = (int)(h % (nx + 1)), k = (int)(h / (nx + 1));
      double v;
      if (j == 0) v = gcat(0, k);
      else if (j == nx) v = gcat(nx - 1, k);
      else v = 0.5 * (gcat(j - 1, k) + gcat(j, k));
      gcsx[(size_t)k * (nx + 1) + j] = v;
    } else {
      const long long h = g - ncell - nsx;     // grav_coeff_stag_y(nx, ny+1)
      const int j = (int)(h % nx), k = (int)(h / nx);
      double v;
      if (k == 0) v = gcat(j, 0);
      else if (k == ny) v = gcat(j, ny - 1);
      else v = 0.5 * (gcat(j, k - 1) + gcat(j, k));
      gcsy[(size_t)k * nx + j] = v;
    }
  }
}

// ============================================================= post step
// The driver's output sweep over the solve cells after each step
// (src/IMEX_SfloW2D.f90:391-442) and its first form after the initial
// check_solve (src/IMEX_SfloW2D.f90:253-309): qp(1) kept for the volume
// print, the running maxima hmax / pdynmax / mod_vel_max, and the
// vulnerability table vuln_table(i_table) = OR over steps of
// (h >= thickness_levels(i_thk)) .AND. (p_dyn >= dyn_pres_levels(i_pdyn)),
// i_table running over i_pdyn fastest.
constexpr int POST_MAX_LEVELS = 10;
constexpr int POST_MAX_WORDS = (POST_MAX_LEVELS * POST_MAX_LEVELS + 31) / 32;

struct PostLevels {
  int n_thk, n_pdyn, n_words, pad_;
  double thk[POST_MAX_LEVELS], pdyn[POST_MAX_LEVELS];
};

struct PostPlanes {
  double* qp_h;     // qp(1,:,:) as the sweep leaves it
  double* hmax;
  double* pdynmax;
  double* mvmax;    // mod_vel_max
  uint32_t* vuln;   // n_words planes; table entry i is bit i%32 of plane i/32
};

template <int NS>
__global__ void __launch_bounds__(128)
    k_post_sweep(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                 const uint8_t* __restrict__ mask, PostPlanes W, PostLevels L, int init) {
  const DevParams& P = Pp;
  constexpr int NV = 4 + NS, NP = 6 + NS;
  const long long ncell = (long long)P.nx * P.ny;
  const size_t N = (size_t)P.plane;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % P.nx), k = (int)(g / P.nx);
    const size_t c = (size_t)k * P.pitch + j;
    if (!mask[c]) continue;
    double qc[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) qc[i] = q[c + i * N];
    if (qc[0] > 0.0) {
      double qpv[NP], pd;
      qc_to_qp<NS>(P, qc, qpv, &pd);
      const double h = qpv[0];
      W.qp_h[c] = h;
      W.hmax[c] = init ? h : fmax_f(W.hmax[c], h);
      const double u = qpv[NV], v = qpv[NV + 1];
      const double mv = sqrt(u * u + v * v);
      if (h > 0.001) {
        W.pdynmax[c] = init ? pd : fmax_f(W.pdynmax[c], pd);
        W.mvmax[c] = init ? mv : fmax_f(W.mvmax[c], mv);
      }
      uint32_t bits[POST_MAX_WORDS] = {0, 0, 0, 0};
      int it = 0;
      for (int a = 0; a < L.n_thk; ++a) {
        const bool thck = h >= L.thk[a];
        for (int b = 0; b < L.n_pdyn; ++b, ++it)
          if (thck && pd >= L.pdyn[b]) bits[it >> 5] |= 1u << (it & 31);
      }
      for (int w = 0; w < L.n_words; ++w) {
        uint32_t* dst = W.vuln + (size_t)w * N + c;
        *dst = init ? bits[w] : (*dst | bits[w]);
      }
    } else {
      W.qp_h[c] = 0.0;
      if (init) {
        W.hmax[c] = 0.0;
        W.pdynmax[c] = 0.0;
      }
    }
  }
}

// The driver's per-step print (src/IMEX_SfloW2D.f90:476-484) before the
// dx*dy factor: SUM(q(1,:,:)), SUM(qp(1,:,:)), COUNT(q(1,:,:) > 1e-7) and
// SUM(q(5:4+n_solid,:,:)).  Per-block partial sums in a fixed order, then
// one block folds them in block order, so the result does not vary from
// run to run.
constexpr int DIAG_THREADS = 256;
template <int NS>
__global__ void __launch_bounds__(DIAG_THREADS)
    k_post_diag(const __grid_constant__ DevParams Pp, const double* __restrict__ q,
                const double* __restrict__ qp_h, double* __restrict__ part) {
  const DevParams& P = Pp;
  const long long ncell = (long long)P.nx * P.ny;
  const size_t N = (size_t)P.plane;
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < ncell;
       g += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(g % P.nx), k = (int)(g / P.nx);
    const size_t c = (size_t)k * P.pitch + j;
    const double h = q[c];
    a[0] += h;
    a[1] += qp_h[c];
    a[2] += (h > 1.0e-7) ? 1.0 : 0.0;
#pragma unroll
    for (int i = 0; i < NS; ++i) a[3] += q[c + (size_t)(4 + i) * N];
  }
  __shared__ double red[4][DIAG_THREADS / 32];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    double x = a[r];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0) red[r][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double x = 0.0;
    for (int w = 0; w < DIAG_THREADS / 32; ++w) x += red[threadIdx.x][w];
    part[(size_t)blockIdx.x * 4 + threadIdx.x] = x;
  }
}

__global__ void k_post_diag_fold(const double* __restrict__ part, int nblocks,
                                 double* __restrict__ out) {
  if (threadIdx.x < 4) {
    double x = 0.0;
    for (int b = 0; b < nblocks; ++b) x += part[(size_t)b * 4 + threadIdx.x];
    out[threadIdx.x] = x;
  }
}

// solve_mask_x / solve_mask_y from solve_mask (src/solver_2d.f90:779-808).
__global__ void k_masks_xy(const __grid_constant__ DevParams Pp, const uint8_t* __restrict__ mask, int8_t* mx,
                           int8_t* my) {
  const DevParams& P = Pp;
  const int nx = P.nx, ny = P.ny;
  long long nX = (long long)(nx + 1) * ny, nY = (long long)nx * (ny + 1);
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < nX + nY;
       g += (long long)gridDim.x * blockDim.x) {
    if (g < nX) {
      int j = (int)(g % (nx + 1)), k = (int)(g / (nx + 1));
      bool m = (j > 0 && mask[(size_t)k * P.pitch + j - 1]) || (j < nx && mask[(size_t)k * P.pitch + j]);
      mx[g] = m ? 1 : 0;
    } else {
      long long h = g - nX;
      int j = (int)(h % nx), k = (int)(h / nx);
      bool m = (k > 0 && mask[(size_t)(k - 1) * P.pitch + j]) || (k < ny && mask[(size_t)k * P.pitch + j]);
      my[h] = m ? 1 : 0;
    }
  }
}

}  // namespace IMEX_TU_NS
}  // namespace imex
