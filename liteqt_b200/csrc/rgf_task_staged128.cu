// rgf_task_staged128.cu -- RGF task function for nb = 128: staged GEMM, blocked Gauss-Jordan.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_staged128(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<StagedOps<128>>(p, t, slot, sm, dyn);
}

}  // namespace rgf
