// rgf_fp64.cu -- the persistent complex FP64 RGF kernel (the drop-in form of
// green_RGF_RS, src/green_rgf.f90:3950-4164, and its adjoint).
//
// One launch drains a work queue of (device, k, E) tasks of any mix of block
// sizes nb and chain lengths nx: a CTA pops a task, looks up the kernel
// variant chosen for the task's nb (staged GEMM + blocked inverse for the
// benchmark sizes, register-direct GEMM for any other multiple of 8; the
// host may override the choice per nb, see rgf_autotune) and calls that
// variant's task function, which runs the whole per-energy chain with the
// CTA's 256 threads (rgf_solver.cuh).  The queue order is set by the host
// (longest tasks first), so the tail of the launch holds the short tasks.
#include <cstdio>

#include "rgf_device.cuh"
#include "rgf_internal.h"
#include "rgf_tasks.h"

namespace rgf {

namespace {

__global__ void __launch_bounds__(kThreads, 2) rgf_solver_kernel(KParams p) {
  extern __shared__ __align__(16) double2 dyn_smem[];
  __shared__ Smem sm;
  double2* slot = p.work + (size_t)blockIdx.x * p.slot_elems;
  for (;;) {
    if (threadIdx.x == 0) sm.task = atomicAdd(p.queue, 1);
    __syncthreads();
    const int64_t q = sm.task;
    __syncthreads();
    if (q >= p.n_tasks) break;
    const int64_t t = p.order ? p.order[q] : q;
    const int dev = p.adj ? p.adj[t].dev : (p.wtasks ? p.wtasks[t].dev : p.tasks[t].dev);
    const int64_t n = p.devs[dev].nm, nx = p.devs[dev].nx;
    int v = KV_NONE;
    if (n >= 8 && n <= kMaxNb && n % 8 == 0) v = p.variant[n / 8];
    const bool staged_ok = (v == KV_STAGED32 && n == 32) || (v == KV_STAGED64 && n == 64) ||
                           (v == KV_STAGED128 && n == 128) || (v == KV_STAGED256 && n == 256);
    const bool generic_ok = v == KV_GENERIC11 || ((v == KV_GENERIC12 || v == KV_GENERIC22) && n % 16 == 0);
    if (!(staged_ok || generic_ok) || nx < 2 || slot_elems_for(n, nx) > p.slot_elems) {
      if (p.info && threadIdx.x == 0) p.info[t].status = RGF_ST_BAD_TASK;
      continue;
    }
    switch (v) {
      case KV_STAGED32: task_staged32(p, t, slot, sm, dyn_smem); break;
      case KV_STAGED64: task_staged64(p, t, slot, sm, dyn_smem); break;
      case KV_STAGED128: task_staged128(p, t, slot, sm, dyn_smem); break;
      case KV_STAGED256: task_staged256(p, t, slot, sm, dyn_smem); break;
      case KV_GENERIC11: task_generic11(p, t, slot, sm, dyn_smem); break;
      case KV_GENERIC12: task_generic12(p, t, slot, sm, dyn_smem); break;
      default: task_generic22(p, t, slot, sm, dyn_smem); break;
    }
  }
}

}  // namespace

int default_variant(int nb) {
  if (nb < 8 || nb > kMaxNb || nb % 8 != 0) return KV_NONE;
  switch (nb) {
    case 32: return KV_STAGED32;
    case 64: return KV_STAGED64;
    case 128: return KV_STAGED128;
    case 256: return KV_STAGED256;
    default: break;
  }
  if (nb % 16 == 0 && nb >= 64) return KV_GENERIC22;
  if (nb % 16 == 0) return KV_GENERIC12;
  return KV_GENERIC11;
}

bool variant_ok(int v, int nb) {
  if (nb < 8 || nb > kMaxNb || nb % 8 != 0) return false;
  switch (v) {
    case KV_STAGED32: return nb == 32;
    case KV_STAGED64: return nb == 64;
    case KV_STAGED128: return nb == 128;
    case KV_STAGED256: return nb == 256;
    case KV_GENERIC11: return true;
    case KV_GENERIC12:
    case KV_GENERIC22: return nb % 16 == 0;
    default: return false;
  }
}

const char* variant_name(int v) {
  static const char* names[KV_COUNT] = {"staged32", "staged64", "staged128", "staged256",
                                        "generic1x1", "generic1x2", "generic2x2"};
  return (v >= 0 && v < KV_COUNT) ? names[v] : "none";
}

size_t variant_smem(int v, int nb) {
  return (v >= KV_STAGED32 && v <= KV_STAGED256) ? smem_staged(nb) : smem_generic(nb);
}

void set_default_variants(KParams& p) {
  for (int i = 0; i < kVariantSlots; i++) p.variant[i] = (int8_t)default_variant(i * 8);
}

int solver_threads() { return kThreads; }

int solver_blocks_per_sm(size_t smem) {
  int nblk = 0;
  cudaFuncSetAttribute(rgf_solver_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nblk, rgf_solver_kernel, kThreads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return nblk > 0 ? nblk : 1;
}

cudaError_t launch_solver(const KParams& p, int grid, size_t smem, cudaStream_t st, bool set_attr) {
  if (set_attr) {
    cudaError_t e = cudaFuncSetAttribute(rgf_solver_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  rgf_solver_kernel<<<grid, kThreads, smem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace rgf
