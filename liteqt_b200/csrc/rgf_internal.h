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
  const double2* Sii;      // overlap blocks (green_RGF_CMS), or NULL = identity
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

// Block-operation policies ("kernel variants") a task can run with:
// staged = shared-memory-staged GEMM + blocked inverse for one block size;
// generic = register-direct GEMM with TM x TN warp tiles for any multiple of 8.
enum KVariant : int {
  KV_NONE = -1,
  KV_STAGED32 = 0, KV_STAGED64, KV_STAGED128, KV_STAGED256,
  KV_GENERIC11, KV_GENERIC12, KV_GENERIC22,
  KV_COUNT
};
constexpr int kVariantSlots = kMaxNb / 8 + 1;  // indexed by nb / 8

// One screened-interaction task (green_rgf_calc_w): the device's Vii / V1i
// sit in DDev's Hii / H1i; polarization inputs and W outputs here.
struct DWTask {
  int32_t dev;
  int32_t pad;
  const double2* PL;
  const double2* PG;
  const double2* PR;
  double2* WL;
  double2* WG;
  double2* WR;
  double2* WRi1;   // blocks 0..nx-2, or NULL
};

struct KParams {
  KOpts o;
  const DDev* devs;
  const DTask* tasks;
  int64_t n_tasks;
  const int32_t* order;    // task order of the queue (longest first), or NULL
  int32_t* queue;          // work-queue counter (zeroed before launch)
  double2* work;           // workspace: one slot per resident CTA
  int64_t slot_elems;      // complex elements per slot (>= slot_elems_for(nb, nx) of every task)
  DInfo* info;             // per task
  int32_t* progress;       // per task, or NULL: blocks whose outputs are written, counted from
                           // the last (host-mapped; the pipelined output copies follow it)
  const DAdj* adj;         // non-null: run the adjoint instead of the drop-in solve
  const DWTask* wtasks;    // non-null: run W solves (green_rgf_calc_w)
  int8_t variant[kVariantSlots];  // kernel variant per block size (nb / 8), KV_NONE = unsupported
};

// Number of named scratch blocks in a slot besides Gl[nx], Gln[nx].
constexpr int kNumTemps = 32;

__host__ __device__ inline int64_t slot_elems_for(int64_t nb, int64_t nx) {
  return (2 * nx + kNumTemps) * nb * nb;
}

// Variant selection (rgf_fp64.cu).
int default_variant(int nb);                 // KV_NONE if nb is unsupported
bool variant_ok(int variant, int nb);
const char* variant_name(int variant);
size_t variant_smem(int variant, int nb);    // dynamic shared memory of a CTA
void set_default_variants(KParams& p);
// Max resident CTAs per SM of the solver kernel with this much dynamic
// shared memory (occupancy query).
int solver_blocks_per_sm(size_t smem);
// Launch the persistent solver over all tasks of p (any mix of block sizes).
// set_attr = false skips raising the kernel's dynamic shared-memory limit
// (inside a stream capture, after solver_blocks_per_sm(smem) has done it).
cudaError_t launch_solver(const KParams& p, int grid, size_t smem, cudaStream_t stream,
                          bool set_attr = true);
int solver_threads();

// Mixed-precision form (rgf_mixed.cu): nb = 128, one CTA per SM.
size_t mixed_smem();                          // dynamic shared memory of a CTA
int64_t mixed_slot_elems(int64_t nx);         // complex elements of one CTA's slot
cudaError_t launch_mixed(const KParams& p, int grid, cudaStream_t stream, bool set_attr = true);
// Batched block operations on nb = 128 blocks, one CTA per block (grid-stride):
// mode 0 split-integer product with ns slices (0 = all), 1 FP64 product,
// 2 refined inverse, 3 FP64 inverse; ws = 5 blocks per CTA; status per block
// or NULL.
cudaError_t launch_block_mixed(int mode, int ns, const double2* A, int cA, const double2* B, int cB,
                               double2* C, int64_t count, double2* ws, int grid, int32_t* status,
                               cudaStream_t stream);
// FP64 inverse of nb = 32, 64 or 128 blocks (the plain form's kernels).
cudaError_t launch_block_fp64_inv(int nb, const double2* X, double2* Xi, int64_t count, double2* ws, int grid,
                                  int32_t* status, cudaStream_t stream);

// Per-context state owned by another module (one slot): a pointer and the
// function that frees it when the context is destroyed.
void* ctx_ext_cache(rgf_ctx* c);
void ctx_set_ext_cache(rgf_ctx* c, void* cache, void (*free_fn)(void*));

}  // namespace rgf
