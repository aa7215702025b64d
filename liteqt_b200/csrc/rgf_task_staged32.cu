// rgf_task_staged32.cu -- RGF task function for nb = 32: staged GEMM, Gauss-Jordan in shared memory.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_staged32(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<StagedOps<32>>(p, t, slot, sm, dyn);
}

size_t smem_staged(int nb) {
  switch (nb) {
    case 32: return StagedOps<32>::smem_bytes(nb);
    case 64: return StagedOps<64>::smem_bytes(nb);
    case 128: return StagedOps<128>::smem_bytes(nb);
    case 256: return StagedOps<256>::smem_bytes(nb);
    default: return 0;
  }
}

}  // namespace rgf
