// Set-up on the device: the DEM sampled at the cell centres
// (src/geometry_2d.f90:320-342 with interp_2d_nodata/interp_2d_scalar,
// :1174-1296), the fraction of each cell inside an elliptical source or
// collapse (compute_cell_fract, :1678-1773) and the area-weighted regridding
// of a restart raster onto the grid (regrid_scalar, :1491-1534, called from
// src/inpout_2d.f90:5205-5246).  Every value comes from the same sequence of
// IEEE operations as the reference's expressions (no contraction), so the
// results equal a CPU evaluation of those expressions bit for bit.
#pragma once

#include <cstdint>

#include "imex_device.cuh"

namespace imex {

// The computational grid as init_grid lays it out: x_stag(J) = x0+(J-1)*dx,
// x_comp(J) = (x_stag(J)+x_stag(J+1))/2 (src/geometry_2d.f90:294-320).
struct SetupGrid {
  int nx, ny;
  double x0, y0, dx, dy;
};

__device__ __forceinline__ double sg_x_comp(const SetupGrid& G, int j) {  // j 0-based
  return 0.5 * ((G.x0 + (double)j * G.dx) + (G.x0 + (double)(j + 1) * G.dx));
}
__device__ __forceinline__ double sg_y_comp(const SetupGrid& G, int k) {
  return 0.5 * ((G.y0 + (double)k * G.dy) + (G.y0 + (double)(k + 1) * G.dy));
}

// A DEM as topography_profile: node coordinates x1(ncols), y1(nrows) and
// heights z(ncols,nrows), column-major, row 1 the southernmost
// (src/inpout_2d.f90:3572-3605).
struct DemView {
  int ncols, nrows;
  const double* x1;
  const double* y1;
  const double* z;
  double nodata;
};

// Error bits of the set-up kernels.
constexpr int SETUP_ERR_OUTSIDE = 1;   // a cell centre below/left of the DEM's first node
constexpr int SETUP_ERR_NONFINITE = 2; // an index from a non-finite coordinate

// FLOOR(v) + 1 as the reference's 1-based index; false when v is not finite
// or out of the int range.
__device__ __forceinline__ bool floor_index(double v, int& out) {
  if (!(v > -1.0e9 && v < 1.0e9)) return false;
  out = (int)floor(v) + 1;
  return true;
}

// interp_2d_nodata (on the heights as read) and interp_2d_scalar (on the
// heights clamped at 0: topography_profile(3,:,:) = MAX(0, ...)) at every
// cell centre.  B_cent and B_nodata are (nx, ny) column-major.
__global__ void __launch_bounds__(256)
    k_dem_to_grid(SetupGrid G, DemView D, double* __restrict__ B_cent,
                  int8_t* __restrict__ B_nodata, int* __restrict__ err) {
  const long long n = (long long)G.nx * G.ny;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(c % G.nx), k = (int)(c / G.nx);
    const double x2 = sg_x_comp(G, j), y2 = sg_y_comp(G, k);
    int ix = 1, iy = 1;
    double ax = 0.0, ay = 0.0;
    bool ok = true;
    if (D.ncols > 1) {
      ok &= floor_index((x2 - D.x1[0]) / (D.x1[1] - D.x1[0]), ix);
      ix = min(ix, D.ncols - 1);
    }
    if (D.nrows > 1) {
      ok &= floor_index((y2 - D.y1[0]) / (D.y1[1] - D.y1[0]), iy);
      iy = min(iy, D.nrows - 1);
    }
    if (!ok || ix < 1 || iy < 1) {
      atomicOr(err, ok ? SETUP_ERR_OUTSIDE : SETUP_ERR_NONFINITE);
      B_cent[c] = 0.0;
      B_nodata[c] = 0;
      continue;
    }
    if (D.ncols > 1) ax = (D.x1[ix] - x2) / (D.x1[ix] - D.x1[ix - 1]);
    if (D.nrows > 1) ay = (D.y1[iy] - y2) / (D.y1[iy] - D.y1[iy - 1]);
    // z(ix,iy) in the reference's 1-based column-major indexing
    const size_t i00 = (size_t)(ix - 1) + (size_t)(iy - 1) * D.ncols;
    const double* z = D.z;
    const double nd = D.nodata;
    bool nod;
    double f2;
    auto zc = [&](size_t i) { return fmax_f(0.0, z[i]); };   // MAX(0, z)
    if (D.ncols == 1) {
      const size_t i01 = i00 + D.ncols;
      nod = (z[i00] == nd) || (z[i01] == nd);
      f2 = ay * zc(i00) + (1.0 - ay) * zc(i01);
    } else if (D.nrows == 1) {
      const size_t i10 = i00 + 1;
      nod = (z[i00] == nd) || (z[i10] == nd);
      f2 = ax * zc(i00) + (1.0 - ax) * zc(i10);
    } else {
      const size_t i01 = i00 + D.ncols, i10 = i00 + 1, i11 = i01 + 1;
      nod = (z[i00] == nd) || (z[i01] == nd) || (z[i10] == nd) || (z[i11] == nd);
      f2 = ax * (ay * zc(i00) + (1.0 - ay) * zc(i01)) +
           (1.0 - ax) * (ay * zc(i10) + (1.0 - ay) * zc(i11));
    }
    B_cent[c] = f2;
    B_nodata[c] = nod ? 1 : 0;
  }
}

// compute_cell_fract: for each cell of the candidate rectangle (cells whose
// box meets the source's bounding square), the share of the 200x200 subgrid
// points inside the ellipse, as REAL(count)/n_points2 in single precision.
// One block per cell; xsub/ysub are the 200 subgrid offsets in x and y.
constexpr int CF_POINTS = 200;
constexpr int CF_THREADS = 256;

struct CellFractArgs {
  SetupGrid G;
  int j_lo, k_lo, n_j, n_k;  // candidate rectangle (0-based)
  double xs, ys, rs2, r2s2, cos_a, sin_a;
};

__global__ void __launch_bounds__(CF_THREADS)
    k_cell_fract(CellFractArgs A, const double* __restrict__ xsub,
                 const double* __restrict__ ysub, double* __restrict__ out) {
  __shared__ double sx[CF_POINTS], sy[CF_POINTS];
  __shared__ int warp_sum[CF_THREADS / 32];
  for (int i = threadIdx.x; i < CF_POINTS; i += CF_THREADS) {
    sx[i] = xsub[i];
    sy[i] = ysub[i];
  }
  __syncthreads();
  const long long ncand = (long long)A.n_j * A.n_k;
  for (long long b = blockIdx.x; b < ncand; b += gridDim.x) {
    const int j = A.j_lo + (int)(b % A.n_j), k = A.k_lo + (int)(b / A.n_j);
    const double xc = sg_x_comp(A.G, j), yc = sg_y_comp(A.G, k);
    int cnt = 0;
    for (int p = threadIdx.x; p < CF_POINTS * CF_POINTS; p += CF_THREADS) {
      const double X = (xc + sx[p % CF_POINTS]) - A.xs;
      const double Y = (yc + sy[p / CF_POINTS]) - A.ys;
      const double u = X * A.cos_a + Y * A.sin_a;
      const double v = -(X * A.sin_a) + Y * A.cos_a;
      if ((u * u) / A.rs2 + (v * v) / A.r2s2 <= 1.0) ++cnt;
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, off);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < CF_THREADS / 32; ++w) tot += warp_sum[w];
      const float fr = (float)tot / (float)(CF_POINTS * CF_POINTS);
      out[(size_t)j + (size_t)k * A.G.nx] = (double)fr;
    }
    __syncthreads();
  }
}

// regrid_scalar for every cell: xl..xr = x0+(j-1)*cell_size .. x0+j*cell_size
// (the restart loop uses cell_size, src/inpout_2d.f90:5217-5227); the input
// raster's edges xin(ncols+1), yin(nrows+1); values equal to `nodata` read
// as 0.  Bounds as in the reference: ix2 <= ncols (SIZE(xin)-1), iy2 <=
// nrows+1 (SIZE(yin)).
struct RegridArgs {
  int nx, ny;
  double x0, y0, cell_size;
  int ncols, nrows;
  double nodata;
};

__device__ __forceinline__ bool ceil_int(double v, int& out) {
  if (!(v > -1.0e9 && v < 1.0e9)) return false;
  out = (int)ceil(v);
  return true;
}

__global__ void __launch_bounds__(256)
    k_regrid(RegridArgs A, const double* __restrict__ xin, const double* __restrict__ yin,
             const double* __restrict__ fin, double* __restrict__ fout, int* __restrict__ err) {
  const long long n = (long long)A.nx * A.ny;
  const double dX = xin[1] - xin[0], dY = yin[1] - yin[0];
  const int nXin = A.ncols, nYin = A.nrows + 1;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(c % A.nx) + 1, k = (int)(c / A.nx) + 1;   // 1-based
    const double xl = A.x0 + (double)(j - 1) * A.cell_size;
    const double xr = A.x0 + (double)j * A.cell_size;
    const double yl = A.y0 + (double)(k - 1) * A.cell_size;
    const double yr = A.y0 + (double)k * A.cell_size;
    int a, b, cc, d;
    if (!ceil_int((xl - xin[0]) / dX, a) || !ceil_int((xr - xin[0]) / dX, b) ||
        !ceil_int((yl - yin[0]) / dY, cc) || !ceil_int((yr - yin[0]) / dY, d)) {
      atomicOr(err, SETUP_ERR_NONFINITE);
      fout[c] = 0.0;
      continue;
    }
    const int ix1 = max(1, a), ix2 = min(nXin, b + 1);
    const int iy1 = max(1, cc), iy2 = min(nYin, d + 1);
    double f = 0.0;
    for (int ix = ix1; ix <= ix2 - 1; ++ix) {
      const double ax = (fmin_f(xr, xin[ix]) - fmax_f(xl, xin[ix - 1])) / (xr - xl);
      for (int iy = iy1; iy <= iy2 - 1; ++iy) {
        const double ay = (fmin_f(yr, yin[iy]) - fmax_f(yl, yin[iy - 1])) / (yr - yl);
        double v = fin[(size_t)(ix - 1) + (size_t)(iy - 1) * A.ncols];
        if (v == A.nodata) v = 0.0;
        f = f + ax * ay * v;
      }
    }
    fout[c] = f;
  }
}

}  // namespace imex
