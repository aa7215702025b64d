// rgf_tasks.h -- the task functions, one per kernel variant, each compiled in
// its own translation unit (rgf_task_*.cu) and linked into the persistent
// kernel by relocatable device code.
#pragma once
#include "rgf_device.cuh"
#include "rgf_internal.h"

namespace rgf {

// Shared-memory state of one CTA, owned by the kernel and passed to the task
// functions.
struct Smem {
  SmemInv inv;
  SmemRed red;
  int64_t task;
};

__device__ void task_staged32(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_staged64(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_staged128(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_staged256(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_generic11(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_generic12(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);
__device__ void task_generic22(const KParams& p, int64_t t, double2* slot, Smem& sm, double2* dyn);

// Dynamic shared memory of each variant (host).
size_t smem_staged(int nb);
size_t smem_generic(int nb);

}  // namespace rgf
