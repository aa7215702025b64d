// rgf_task_staged64.cu -- RGF task function for nb = 64: staged GEMM, Gauss-Jordan in shared memory.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_staged64(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<StagedOps<64>>(p, t, slot, sm, dyn);
}

}  // namespace rgf
