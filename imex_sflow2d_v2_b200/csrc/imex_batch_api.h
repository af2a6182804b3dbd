// imex_batch_api.h -- host interface between the library's translation
// units and the batched ensemble step (imex_batch.cu).  Plain types only:
// each translation unit has its own (identical) copy of the device types.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace imex_batch {

// One member, from its context: the host copies of its DevParams and
// NewtonWork (their byte sizes checked against the batch unit's), its device
// planes, and its place in the ensemble's tile numbering.
struct MemberSrc {
  const void* params;
  size_t params_bytes;
  const void* newton_work;
  size_t newton_work_bytes;
  double* q;
  double* X;
  uint8_t* mask;
  const uint8_t* cellinfo;
  const double* release;
  const double *Bx, *By, *Bxx, *Bxy, *Byy, *gc, *dgc, *gcsx, *gcsy;
  const void* ring;
  double *erodible, *deposit, *erosion, *Bcent;
  void* clk;
  int tiles_x;
  int exchange;
  long long tile0;
};

// Bytes of one member record in the device member table.
size_t member_bytes();
// Writes member record `s` into `dst` (member_bytes() bytes of host
// memory); false if the type sizes of the two units disagree.
bool fill_member(void* dst, const MemberSrc& s);

// One batched step of all members on `stream`.
struct Launch {
  void* members;                  // device member table
  int n_members;
  int ns;                         // solid classes (the same for all members)
  int shape;                      // 0: 32x8, 1: 16x16, 2: 32x4 tiles
  const uint32_t* tile_member;    // global tile -> member
  uint32_t* active;               // active-tile list
  unsigned int* n_active;
  unsigned long long* list_off;   // n_members + 1 list offsets
  long long n_tiles;
  int any_exchange;               // some member runs erosion/deposition
  int sms;                        // multiprocessors of the device
  cudaStream_t stream;
};
// Enqueues the step; *launches receives the number of kernels.
cudaError_t enqueue_step(const Launch& L, int* launches);

}  // namespace imex_batch
