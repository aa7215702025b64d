// rgf_task_staged256.cu -- RGF task function for nb = 256: staged GEMM, blocked Gauss-Jordan.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_staged256(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<StagedOps<256>>(p, t, slot, sm, dyn);
}

}  // namespace rgf
