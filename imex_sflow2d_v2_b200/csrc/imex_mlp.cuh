// imex_mlp.cuh -- the small network that proposes the Newton starting point
// of stage 2 (learned warm start), with its own training kernels.
//
// Shape: 12 inputs -> 3 hidden layers of 64 (SiLU) -> 2 outputs.  Inputs are
// padded to 16 and outputs to 8 so that every layer is a whole number of
// m16n8k16 tensor-core tiles.  Weights are kept in FP32 (the Adam master copy)
// and in BF16 (the operands of the forward pass); products accumulate in FP32.
//
// Forward (inference and training): one warp carries 16 samples through the
// four layers with mma.sync.m16n8k16 BF16 tiles; a layer's FP32 result tile
// is, element for element, the A operand of the next layer once rounded to
// BF16, so activations stay in registers between layers.
// Backward (training): FP32 on the CUDA cores from the activations the
// forward pass leaves in shared memory; per-block gradient sums in shared
// memory, one atomic add per parameter and block into the global gradient.
// Adam updates the FP32 master weights and refreshes the BF16 copies.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace imex {
inline namespace IMEX_TU_NS {
namespace mlp {

constexpr int IN = 12, IN_P = 16;   // features (padded)
constexpr int HID = 64;
constexpr int OUT = 2, OUT_P = 8;   // outputs (padded)
// FP32 parameter vector: W0[IN_P][HID] b0[HID] W1[HID][HID] b1 W2[HID][HID] b2
// W3[HID][OUT_P] b3[OUT_P]; row index = input, column = output.
constexpr int OFF_W0 = 0;
constexpr int OFF_B0 = OFF_W0 + IN_P * HID;
constexpr int OFF_W1 = OFF_B0 + HID;
constexpr int OFF_B1 = OFF_W1 + HID * HID;
constexpr int OFF_W2 = OFF_B1 + HID;
constexpr int OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_W3 = OFF_B2 + HID;
constexpr int OFF_B3 = OFF_W3 + HID * OUT_P;
constexpr int NPARAM = OFF_B3 + OUT_P;
// BF16 weight copies (biases stay FP32)
constexpr int BOFF_W0 = 0;
constexpr int BOFF_W1 = BOFF_W0 + IN_P * HID;
constexpr int BOFF_W2 = BOFF_W1 + HID * HID;
constexpr int BOFF_W3 = BOFF_W2 + HID * HID;
constexpr int NBW = BOFF_W3 + HID * OUT_P;

constexpr int WARPS = 4;               // per block
constexpr int SAMPLES = 16 * WARPS;    // per block and pass

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
  float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B operand of tile (k-step ks, n-tile nt) from a BF16 [K][N] row-major
// matrix in shared memory: rows k = 16ks + 2t + {0,1} (+8), column 8nt + g.
__device__ __forceinline__ void load_b(const __nv_bfloat16* W, int N, int ks, int nt, int g,
                                       int t, uint32_t& b0, uint32_t& b1) {
  const int n = 8 * nt + g, k = 16 * ks + 2 * t;
  __nv_bfloat162 v0, v1;
  v0.x = W[(k + 0) * N + n];
  v0.y = W[(k + 1) * N + n];
  v1.x = W[(k + 8) * N + n];
  v1.y = W[(k + 9) * N + n];
  b0 = *reinterpret_cast<uint32_t*>(&v0);
  b1 = *reinterpret_cast<uint32_t*>(&v1);
}

// Per-warp activation record for the backward pass (FP32; a* hold the
// BF16-rounded values that entered the next layer).
struct WarpAct {
  float a0[16][IN_P];
  float z1[16][HID], a1[16][HID];
  float z2[16][HID], a2[16][HID];
  float z3[16][HID], a3[16][HID];
  float y[16][OUT_P];
};

// Forward pass of 16 samples by one warp.  x: the warp's 16 normalised
// inputs, row-major [16][IN] (FP32, any memory the warp can read; rows with
// valid == false are fed as zeros).  W: BF16 weights, bias: FP32 parameter
// vector (both in shared memory).  y: [16][OUT] outputs (lane-distributed
// writes); rec: activation record, or nullptr for inference.
__device__ void forward16(const float* x, int nvalid, const __nv_bfloat16* W, const float* prm,
                          float* y, int ldy, WarpAct* rec) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // layer 0 A operand: rows g, g+8; cols 2t,2t+1 (k 0..7) and +8
  uint32_t a[4][4];  // A operands of the next layer, per 16-wide k-step
  {
    float v[2][4];
    for (int r = 0; r < 2; ++r) {
      const int s = g + 8 * r;
      for (int h = 0; h < 2; ++h)
        for (int i = 0; i < 2; ++i) {
          const int col = 2 * t + 8 * h + i;
          float xv = (s < nvalid && col < IN) ? x[s * IN + col] : 0.0f;
          v[r][2 * h + i] = xv;
          if (rec) rec->a0[s][col] = bf16r(xv);
        }
    }
    a[0][0] = pack_bf16(v[0][0], v[0][1]);
    a[0][1] = pack_bf16(v[1][0], v[1][1]);
    a[0][2] = pack_bf16(v[0][2], v[0][3]);
    a[0][3] = pack_bf16(v[1][2], v[1][3]);
  }
  int ksteps = 1;
  const __nv_bfloat16* Wl[4] = {W + BOFF_W0, W + BOFF_W1, W + BOFF_W2, W + BOFF_W3};
  const float* bl[4] = {prm + OFF_B0, prm + OFF_B1, prm + OFF_B2, prm + OFF_B3};
  for (int layer = 0; layer < 3; ++layer) {
    float acc[8][4];
    for (int nt = 0; nt < 8; ++nt) {
      const float b0v = bl[layer][8 * nt + 2 * t], b1v = bl[layer][8 * nt + 2 * t + 1];
      acc[nt][0] = b0v;
      acc[nt][1] = b1v;
      acc[nt][2] = b0v;
      acc[nt][3] = b1v;
      for (int ks = 0; ks < ksteps; ++ks) {
        uint32_t bb0, bb1;
        load_b(Wl[layer], HID, ks, nt, g, t, bb0, bb1);
        mma_bf16(acc[nt], a[ks], bb0, bb1);
      }
    }
    // SiLU; the result tiles become the next layer's A operands
    for (int nt = 0; nt < 8; ++nt) {
      float s[4];
      for (int e = 0; e < 4; ++e) s[e] = silu(acc[nt][e]);
      if (rec) {
        float(*z)[HID] = layer == 0 ? rec->z1 : (layer == 1 ? rec->z2 : rec->z3);
        float(*av)[HID] = layer == 0 ? rec->a1 : (layer == 1 ? rec->a2 : rec->a3);
        for (int e = 0; e < 4; ++e) {
          const int row = g + 8 * (e >> 1), col = 8 * nt + 2 * t + (e & 1);
          z[row][col] = acc[nt][e];
          av[row][col] = bf16r(s[e]);
        }
      }
      const int ks = nt >> 1, half = nt & 1;
      a[ks][2 * half + 0] = pack_bf16(s[0], s[1]);
      a[ks][2 * half + 1] = pack_bf16(s[2], s[3]);
    }
    ksteps = 4;
  }
  // output layer: one n-tile of 8 (2 used)
  float out[4];
  {
    const float b0v = bl[3][2 * t], b1v = bl[3][2 * t + 1];
    out[0] = b0v;
    out[1] = b1v;
    out[2] = b0v;
    out[3] = b1v;
    for (int ks = 0; ks < 4; ++ks) {
      uint32_t bb0, bb1;
      load_b(Wl[3], OUT_P, ks, 0, g, t, bb0, bb1);
      mma_bf16(out, a[ks], bb0, bb1);
    }
  }
  for (int e = 0; e < 4; ++e) {
    const int row = g + 8 * (e >> 1), col = 2 * t + (e & 1);
    if (rec) rec->y[row][col] = out[e];
    if (y && col < OUT && row < nvalid) y[row * ldy + col] = out[e];
  }
}

// Loads the BF16 weights and FP32 parameters into shared memory.
__device__ __forceinline__ void load_net(const __nv_bfloat16* gW, const float* gP,
                                         __nv_bfloat16* sW, float* sP) {
  for (int i = threadIdx.x; i < NBW; i += blockDim.x) sW[i] = gW[i];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sP[i] = gP[i];
}

constexpr size_t SMEM_NET = NBW * sizeof(__nv_bfloat16) + NPARAM * sizeof(float);

// Inference over n samples: x [n][IN], y [n][OUT] (normalised values).
__global__ void __launch_bounds__(32 * WARPS)
    k_mlp_predict(const __nv_bfloat16* __restrict__ gW, const float* __restrict__ gP,
                  const float* __restrict__ x, float* __restrict__ y, long long n) {
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
  float* sP = reinterpret_cast<float*>(smem + NBW * sizeof(__nv_bfloat16));
  load_net(gW, gP, sW, sP);
  __syncthreads();
  const int warp = threadIdx.x >> 5;
  for (long long s0 = ((long long)blockIdx.x * WARPS + warp) * 16; s0 < n;
       s0 += (long long)gridDim.x * WARPS * 16) {
    const int nvalid = (int)((n - s0) < 16 ? (n - s0) : 16);
    forward16(x + s0 * IN, nvalid, sW, sP, y + s0 * OUT, OUT, nullptr);
  }
}

// One training pass over the samples [base, base + n_batch): mean squared
// error over samples and the OUT outputs; gradients added to grad (FP32),
// the summed squared error to *loss_sum.
__global__ void __launch_bounds__(32 * WARPS)
    k_mlp_grad(const __nv_bfloat16* __restrict__ gW, const float* __restrict__ gP,
               const float* __restrict__ x, const float* __restrict__ yt, long long n_batch,
               float inv_count, float* __restrict__ grad, float* __restrict__ loss_sum) {
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
  float* sP = reinterpret_cast<float*>(smem + NBW * sizeof(__nv_bfloat16));
  float* sG = sP + NPARAM;                                      // block gradient sums
  WarpAct* act = reinterpret_cast<WarpAct*>(sG + NPARAM);       // one per warp
  load_net(gW, gP, sW, sP);
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) sG[i] = 0.0f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpAct& A = act[warp];
  float lsum = 0.0f;
  for (long long s0 = ((long long)blockIdx.x * WARPS + warp) * 16; s0 < n_batch;
       s0 += (long long)gridDim.x * WARPS * 16) {
    const int nv = (int)((n_batch - s0) < 16 ? (n_batch - s0) : 16);
    forward16(x + s0 * IN, nv, sW, sP, nullptr, 0, &A);
    __syncwarp();
    // dL/dy for valid samples and the OUT real outputs: (y - t) * 2/count
    __shared__ float dz4s[WARPS][16][OUT_P];
    for (int e = lane; e < 16 * OUT_P; e += 32) {
      const int s = e / OUT_P, o = e % OUT_P;
      float d = 0.0f;
      if (s < nv && o < OUT) {
        const float r = A.y[s][o] - yt[(s0 + s) * OUT + o];
        lsum += r * r;
        d = 2.0f * r * inv_count;
      }
      dz4s[warp][s][o] = d;
    }
    __syncwarp();
    float(*dz4)[OUT_P] = dz4s[warp];
    // output layer: dW3[k][o] = sum_s a3[s][k] dz4[s][o]; db3; da3 -> dz3 (into z3)
    for (int e = lane; e < HID * OUT; e += 32) {
      const int k = e / OUT, o = e % OUT;
      float acc = 0.0f;
      for (int s = 0; s < nv; ++s) acc += A.a3[s][k] * dz4[s][o];
      atomicAdd(&sG[OFF_W3 + k * OUT_P + o], acc);
    }
    if (lane < OUT) {
      float acc = 0.0f;
      for (int s = 0; s < nv; ++s) acc += dz4[s][lane];
      atomicAdd(&sG[OFF_B3 + lane], acc);
    }
    // dz for hidden layer 3: (W3 dz4) * silu'(z3), overwriting z3
    __syncwarp();
    for (int e = lane; e < 16 * HID; e += 32) {
      const int s = e / HID, k = e % HID;
      float d = 0.0f;
      for (int o = 0; o < OUT; ++o) d += __bfloat162float(sW[BOFF_W3 + k * OUT_P + o]) * dz4[s][o];
      A.z3[s][k] = (s < nv) ? d * silu_grad(A.z3[s][k]) : 0.0f;
    }
    __syncwarp();
    // hidden layers 3 -> 2 -> 1
    for (int l = 2; l >= 0; --l) {
      float(*dz)[HID] = l == 2 ? A.z3 : (l == 1 ? A.z2 : A.z1);
      const int in_dim = l == 0 ? IN_P : HID;
      const int offW = l == 2 ? OFF_W2 : (l == 1 ? OFF_W1 : OFF_W0);
      const int offB = l == 2 ? OFF_B2 : (l == 1 ? OFF_B1 : OFF_B0);
      const int boffW = l == 2 ? BOFF_W2 : (l == 1 ? BOFF_W1 : BOFF_W0);
      for (int e = lane; e < in_dim * HID; e += 32) {
        const int k = e / HID, nn = e % HID;
        float acc = 0.0f;
        if (l == 0) {
          for (int s = 0; s < nv; ++s) acc += A.a0[s][k] * dz[s][nn];
        } else {
          float(*ain)[HID] = l == 2 ? A.a2 : A.a1;
          for (int s = 0; s < nv; ++s) acc += ain[s][k] * dz[s][nn];
        }
        atomicAdd(&sG[offW + k * HID + nn], acc);
      }
      for (int nn = lane; nn < HID; nn += 32) {
        float acc = 0.0f;
        for (int s = 0; s < nv; ++s) acc += dz[s][nn];
        atomicAdd(&sG[offB + nn], acc);
      }
      if (l > 0) {
        float(*dzp)[HID] = l == 2 ? A.z2 : A.z1;  // pre-activations of the layer below
        __syncwarp();
        // dz_below = (W_l dz) * silu'(z_below); computed into registers first
        float tmp[16 * HID / 32];
        for (int e = lane, i = 0; e < 16 * HID; e += 32, ++i) {
          const int s = e / HID, k = e % HID;
          float d = 0.0f;
          for (int nn = 0; nn < HID; ++nn)
            d += __bfloat162float(sW[boffW + k * HID + nn]) * dz[s][nn];
          tmp[i] = (s < nv) ? d * silu_grad(dzp[s][k]) : 0.0f;
        }
        __syncwarp();
        for (int e = lane, i = 0; e < 16 * HID; e += 32, ++i) dzp[e / HID][e % HID] = tmp[i];
        __syncwarp();
      }
    }
    __syncwarp();
  }
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
  if (lane == 0) atomicAdd(loss_sum, lsum);
  __syncthreads();
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x)
    if (sG[i] != 0.0f) atomicAdd(&grad[i], sG[i]);
}

constexpr size_t SMEM_GRAD = SMEM_NET + NPARAM * sizeof(float) + WARPS * sizeof(WarpAct);

// Adam step on the FP32 master parameters; clears the gradient.  Padded
// rows/columns stay zero (so are their gradients).
__global__ void k_mlp_adam(float* __restrict__ prm, float* __restrict__ grad, float* __restrict__ m1,
                           float* __restrict__ m2, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NPARAM; i += gridDim.x * blockDim.x) {
    const float gi = grad[i];
    const float m = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = m;
    m2[i] = v;
    const float p = prm[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    prm[i] = p;
    grad[i] = 0.0f;
  }
}

// BF16 copies of the weights from the FP32 parameters.
__global__ void k_mlp_to_bf16(const float* __restrict__ prm, __nv_bfloat16* __restrict__ bw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NBW; i += gridDim.x * blockDim.x) {
    int src;
    if (i < BOFF_W1) src = OFF_W0 + i;
    else if (i < BOFF_W2) src = OFF_W1 + (i - BOFF_W1);
    else if (i < BOFF_W3) src = OFF_W2 + (i - BOFF_W2);
    else src = OFF_W3 + (i - BOFF_W3);
    bw[i] = __float2bfloat16_rn(prm[src]);
  }
}

// Row gather (shuffling the training set once): dst[i] = src[perm[i]].
__global__ void k_gather_rows(const float* __restrict__ src, const long long* __restrict__ perm,
                              float* __restrict__ dst, long long n, int w) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n * w;
       e += (long long)gridDim.x * blockDim.x)
    dst[e] = src[perm[e / w] * w + e % w];
}

}  // namespace mlp
}  // namespace IMEX_TU_NS
}  // namespace imex
