// rgf_internal.h -- structures shared by the host API (rgf_api.cu) and the
// device kernels.  Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rgf.h"

namespace rgf {

constexpr int kMaxNb = 256;  // largest block size (orbitals per block)

// Options as the kernels see them (copied from rgf_opts).
struct KOpts {
  double eta_dev;
  double eta_lead;
  double boltz;
  double sancho_tol;
  int32_t sancho_nmax;
  int32_t consistent;
  int32_t want_T;
  int32_t pad;
};

// One device (Hamiltonian), device pointers only.
struct DDev {
  int64_t nm, nx;
  const double2* Hii;
  const double2* H1i;
  double mu[2];
  double temp[2];
};

// One task, device pointers only (NULL = absent).
struct DTask {
  int32_t dev;
  int32_t pad;
  double E;
  const double2* sig_lesser;
  const double2* sig_r;
  double2* ldos;
  double2* ndens;
  double2* pdens;
  double2* GRi1;
  double2* GLi1;
  double2* GGi1;
  double* cur;
  double* tr;
  double* tre;
  double* T;
};

// Per-task diagnostics (layout identical to rgf_task_info).
struct DInfo {
  int32_t status;
  int32_t sancho_iters_left;
  int32_t sancho_iters_right;
  int32_t n_gemm;
  int32_t n_inv;
  int32_t pad;
};
static_assert(sizeof(DInfo) == sizeof(rgf_task_info), "DInfo layout");

// One adjoint task (ballistic): T(E), dT/dV_l for every block, dT/ds for the
// interior coupling scale.
struct DAdj {
  int32_t dev;
  int32_t pad;
  double E;
  double* T;       // scalar
  double* dTdV;    // nx values
  double* dTds;    // scalar
};

struct KParams {
  KOpts o;
  const DDev* devs;
  const DTask* tasks;
  int64_t n_tasks;
  const int32_t* order;    // task order of the queue (longest first), or NULL
  int32_t* queue;          // work-queue counter (zeroed before launch)
  double2* work;           // workspace: one slot per resident CTA
  int64_t slot_elems;      // complex elements per slot
  int64_t nx_max;          // Gl / Gln capacity per slot
  int32_t nb;              // block size of every task in this launch
  int32_t pad;
  DInfo* info;             // per task
  const DAdj* adj;         // non-null: run the adjoint instead of the drop-in solve
};

// Number of named scratch blocks in a slot besides Gl[nx_max], Gln[nx_max].
constexpr int kNumTemps = 32;

inline int64_t slot_elems_for(int64_t nb, int64_t nx_max) {
  return (2 * nx_max + kNumTemps) * nb * nb;
}

// Launch the FP64 solver over all tasks (all tasks have block size p.nb).
// Returns the CUDA error of the launch.
cudaError_t launch_fp64(const KParams& p, int grid, cudaStream_t stream);
int fp64_threads();
// Max resident CTAs per SM for block size nb (occupancy query).
int fp64_blocks_per_sm(int nb);
size_t fp64_smem_bytes(int nb);

}  // namespace rgf
