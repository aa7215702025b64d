// rgf_task_generic22.cu -- RGF task function for any nb (multiple of 16): register-direct GEMM, 16x16 warp tiles.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_generic22(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<GenericOps<2, 2>>(p, t, slot, sm, dyn);
}

}  // namespace rgf
