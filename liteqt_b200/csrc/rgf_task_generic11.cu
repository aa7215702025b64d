// rgf_task_generic11.cu -- RGF task function for any nb (multiple of 8): register-direct GEMM, 8x8 warp tiles.
#include "rgf_solver.cuh"
#include "rgf_tasks.h"

namespace rgf {

__device__ __noinline__ void task_generic11(const KParams& p, int64_t t, double2* slot, Smem& sm,
                                         double2* dyn) {
  solve_task<GenericOps<1, 1>>(p, t, slot, sm, dyn);
}

size_t smem_generic(int nb) { return GenericOps<1, 1>::smem_bytes(nb); }

}  // namespace rgf
