// imex_batch.cu -- the batched ensemble step (kernels in imex_batch.cuh),
// compiled as its own translation unit so that the library's units build in
// parallel.  Interface: imex_batch_api.h.
#include <cuda_runtime.h>

// namespace of this unit's copy of the kernels (imex_device.cuh)
#define IMEX_TU_NS tu_batch

#include <algorithm>
#include <atomic>
#include <cstring>

#include "imex_batch.cuh"
#include "imex_batch_api.h"

using namespace imex;

namespace imex_batch {

namespace {

// Dynamic shared-memory attributes belong to a device: bit d records that
// they have been set on device d.
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

template <int NS, class TS>
cudaError_t enqueue_ns(const Launch& L, int* launches) {
  MemberDev* M = static_cast<MemberDev*>(L.members);
  const int n = L.n_members, sms = L.sms;
  const size_t smem = kb_flux_smem<NS, TS>();
  static std::atomic<unsigned long long> attr{0};
  if (attr_needed(attr)) {
    cudaError_t e = cudaFuncSetAttribute(kb_flux<NS, TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kb_flux<NS, TS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    attr_done(attr);
  }
  cudaStream_t st = L.stream;
  const int mgrid = (n + 127) / 128;
  const long long tiles = L.n_tiles;
  const int tx = TS::TX, ty = TS::TY;
  auto wave = [&](long long per_sm) { return (int)std::min<long long>(tiles, sms * per_sm); };
  kb_step_begin<<<mgrid, 128, 0, st>>>(M, n, L.n_active);
  kb_mask<TS><<<wave(8), 256, 0, st>>>(M, L.tile_member, tiles, L.active, L.n_active);
  kb_flux<NS, TS><<<wave(flux_min_blocks<NS, TS>()), TS::THREADS, smem, st>>>(
      M, L.tile_member, L.active, L.n_active);
  kb_dt_clip<<<mgrid, 128, 0, st>>>(M, n);
  kb_stage2_first<NS><<<wave(IMEX_FIRST_MINB), STAGE2_THREADS, 0, st>>>(
      M, L.tile_member, L.active, L.n_active, tx, ty);
  for (int pass = 0; pass < 3; ++pass) {
    kb_list_offsets<<<1, 1024, 0, st>>>(M, n, pass, L.list_off);
    if (pass < 2)
      kb_stage2_iter<NS><<<sms * IMEX_STAGE2_MINB, STAGE2_THREADS, 0, st>>>(M, n, L.list_off,
                                                                              pass + 2);
    else
      kb_stage2_tail<NS><<<sms * IMEX_STAGE2_MINB, STAGE2_THREADS, 0, st>>>(M, n, L.list_off);
  }
  kb_stage2_post<NS><<<wave(8), STAGE2_THREADS, 0, st>>>(M, L.tile_member, L.active, L.n_active,
                                                         tx, ty);
  if (L.any_exchange)
    kb_erosion<NS><<<wave(IMEX_EROSION_MINB), 128, 0, st>>>(M, L.tile_member, L.active,
                                                            L.n_active, tx, ty);
  kb_step_end<<<mgrid, 128, 0, st>>>(M, n);
  *launches = 13 + (L.any_exchange ? 1 : 0);
  return cudaGetLastError();
}

template <int NS>
cudaError_t enqueue_shape(const Launch& L, int* launches) {
  switch (L.shape) {
    case 0: return enqueue_ns<NS, Shape32x8>(L, launches);
    case 1: return enqueue_ns<NS, Shape16x16>(L, launches);
    default: return enqueue_ns<NS, Shape32x4>(L, launches);
  }
}

}  // namespace

size_t member_bytes() { return sizeof(MemberDev); }

bool fill_member(void* dst, const MemberSrc& s) {
  if (s.params_bytes != sizeof(DevParams) || s.newton_work_bytes != sizeof(NewtonWork))
    return false;
  MemberDev d;
  std::memset(&d, 0, sizeof(d));
  std::memcpy(&d.P, s.params, sizeof(DevParams));
  std::memcpy(&d.W, s.newton_work, sizeof(NewtonWork));
  d.q = s.q;
  d.X = s.X;
  d.mask = s.mask;
  d.cellinfo = s.cellinfo;
  d.release = s.release;
  d.Bx = s.Bx; d.By = s.By; d.Bxx = s.Bxx; d.Bxy = s.Bxy; d.Byy = s.Byy;
  d.gc = s.gc; d.dgc = s.dgc; d.gcsx = s.gcsx; d.gcsy = s.gcsy;
  d.ring = static_cast<const RingCell*>(s.ring);
  d.erodible = s.erodible; d.deposit = s.deposit; d.erosion = s.erosion; d.Bcent = s.Bcent;
  d.clk = static_cast<DevClock*>(s.clk);
  d.tiles_x = s.tiles_x;
  d.exchange = s.exchange;
  d.tile0 = s.tile0;
  std::memcpy(dst, &d, sizeof(d));
  return true;
}

cudaError_t enqueue_step(const Launch& L, int* launches) {
  switch (L.ns) {
    case 1: return enqueue_shape<1>(L, launches);
    case 2: return enqueue_shape<2>(L, launches);
    case 3: return enqueue_shape<3>(L, launches);
    default: return enqueue_shape<4>(L, launches);
  }
}

}  // namespace imex_batch
