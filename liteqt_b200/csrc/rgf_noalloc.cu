// rgf_noalloc.cu -- the batched FP64 solve without any device allocation.
//
// rgf_solve_energies() keeps its workspace, task tables and staging buffers
// in device memory that the library allocates (cudaMalloc) on first use.
// Some callers cannot allow that: a host code that hands all of HBM to its
// own memory pool at start-up (a framework's caching allocator, or a
// transport solver that preallocates its Green's-function arrays and runs
// close to the memory limit) must not see a library allocate behind its
// back, and a driver that calls the solver inside its energy loop cannot
// take the implicit device-wide synchronisation of cudaMalloc / cudaFree.
// rgf_solve_energies_noalloc() serves them: every array it touches is either
// the caller's (device memory only) or lives in the fixed scratch array
// below, which is part of the library image and is reserved on every GPU
// that loads the library, until the process exits.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "rgf_internal.h"

namespace {

// Fixed scratch: 256 MiB, 256-byte aligned.  Holds the work-queue counter,
// the device descriptor, the task and status tables and the per-CTA solver
// workspace.
constexpr size_t kScratchBytes = size_t(256) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;            // one call at a time per process: calls share the scratch
void* g_scratch_addr[kMaxDevices] = {};

thread_local char g_err[512];

int err(int code, const char* msg) {
  std::snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}

// Device memory of GPU `dev` (managed memory is reachable from every GPU);
// an array on another GPU would be read through a peer address, which
// faults without peer access.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  return a.type == cudaMemoryTypeDevice && a.device == dev;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" const char* rgf_noalloc_last_error(void) { return g_err; }

extern "C" int rgf_solve_energies_noalloc(const rgf_opts* opts, const rgf_device* device,
                                          int64_t nen, const double* E,
                                          const rgf_c16* sigma_lesser, const rgf_c16* sigma_r,
                                          rgf_c16* ldos, rgf_c16* ndens, rgf_c16* pdens,
                                          rgf_c16* GRi1, double* cur, double* tr, double* tre,
                                          double* T, rgf_task_info* info, void* stream) {
  using namespace rgf;
  g_err[0] = 0;
  if (!opts || !device || !E || nen < 1) return err(RGF_E_ARG, "NULL argument or nen < 1");
  if (opts->struct_size != (int32_t)sizeof(rgf_opts)) return err(RGF_E_ARG, "rgf_opts.struct_size mismatch");
  if (opts->precision != RGF_PREC_FP64) return err(RGF_E_UNSUPPORTED, "only RGF_PREC_FP64 is available without allocation");
  const int64_t nm = device->nm, nx = device->nx;
  if (nm < 8 || nm > kMaxNb || nm % 8 != 0) return err(RGF_E_UNSUPPORTED, "nm must be a multiple of 8 in [8, 256]");
  if (nx < 2) return err(RGF_E_ARG, "nx < 2");
  if (!(device->temp[0] > 0.0) || !(device->temp[1] > 0.0)) return err(RGF_E_ARG, "temperature must be > 0");
  const void* arrays[] = {device->Hii, device->H1i, device->Sii, sigma_lesser, sigma_r, ldos, ndens,
                          pdens, GRi1, cur, tr, tre, T};
  if (!device->Hii || !device->H1i) return err(RGF_E_ARG, "Hii / H1i is NULL");
  int cur_dev = -1;
  if (cudaGetDevice(&cur_dev) != cudaSuccess) return err(RGF_E_CUDA, "cudaGetDevice failed");
  if (opts->device != cur_dev) return err(RGF_E_ARG, "opts.device must be the current CUDA device");
  for (const void* a : arrays)
    if (a && !on_device(a, cur_dev))
      return err(RGF_E_ARG, "every array must be device memory of the current device (host arrays would "
                            "need staging buffers)");

  // scratch layout: queue | device | tasks | status | order | per-CTA slots
  const size_t off_dev = 256;
  const size_t off_tasks = off_dev + align256(sizeof(DDev));
  const size_t off_info = off_tasks + align256(sizeof(DTask) * (size_t)nen);
  const size_t off_order = off_info + align256(sizeof(DInfo) * (size_t)nen);
  const size_t off_slots = off_order + align256(sizeof(int32_t) * (size_t)nen);
  const size_t slot_bytes = sizeof(double2) * (size_t)slot_elems_for(nm, nx);
  if (off_slots + slot_bytes > kScratchBytes) {
    std::snprintf(g_err, sizeof(g_err),
                  "problem too large for the %zu MiB no-alloc scratch: nm=%lld nx=%lld nen=%lld needs "
                  "%zu bytes for one solver slot plus %zu bytes of tables",
                  kScratchBytes >> 20, (long long)nm, (long long)nx, (long long)nen, slot_bytes, off_slots);
    return RGF_E_ARG;
  }

  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return err(RGF_E_CUDA, "cudaGetDevice failed");
  if (opts->device != dev) return err(RGF_E_ARG, "opts.device must be the current CUDA device");
  // Set-up, once per device, with that device current: the host-side name of
  // the scratch array is not a device address, so ask the runtime for it.
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return err(RGF_E_CUDA, cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  char* base = (char*)g_scratch_addr[dev];
  cudaStream_t st = (cudaStream_t)stream;

  DDev dd;
  std::memset(&dd, 0, sizeof(dd));
  dd.nm = nm;
  dd.nx = nx;
  dd.Hii = (const double2*)device->Hii;
  dd.H1i = (const double2*)device->H1i;
  dd.Sii = (const double2*)device->Sii;
  for (int i = 0; i < 2; i++) { dd.mu[i] = device->mu[i]; dd.temp[i] = device->temp[i]; }
  const size_t per = (size_t)nm * nm * nx;
  std::vector<DTask> tasks((size_t)nen);
  std::vector<int32_t> order((size_t)nen);
  for (int64_t e = 0; e < nen; e++) {
    DTask& t = tasks[e];
    std::memset(&t, 0, sizeof(t));
    t.E = E[e];
    t.sig_lesser = sigma_lesser ? (const double2*)(sigma_lesser + e * per) : nullptr;
    t.sig_r = sigma_r ? (const double2*)(sigma_r + e * per) : nullptr;
    t.ldos = ldos ? (double2*)(ldos + e * per) : nullptr;
    t.ndens = ndens ? (double2*)(ndens + e * per) : nullptr;
    t.pdens = pdens ? (double2*)(pdens + e * per) : nullptr;
    t.GRi1 = GRi1 ? (double2*)(GRi1 + e * per) : nullptr;
    t.cur = cur ? cur + e * per : nullptr;
    t.tr = tr ? tr + e : nullptr;
    t.tre = tre ? tre + e : nullptr;
    t.T = (opts->want_T && T) ? T + e : nullptr;
    order[e] = (int32_t)e;
  }
#define NA_CUDA(call)                                          \
  do {                                                         \
    const cudaError_t ce = (call);                             \
    if (ce != cudaSuccess) return err(RGF_E_CUDA, cudaGetErrorString(ce)); \
  } while (0)
  // the scratch keeps the previous call's contents: the queue counter and
  // the status words must start at zero
  NA_CUDA(cudaMemsetAsync(base, 0, 256, st));
  NA_CUDA(cudaMemsetAsync(base + off_info, 0, sizeof(DInfo) * (size_t)nen, st));
  NA_CUDA(cudaMemcpyAsync(base + off_dev, &dd, sizeof(DDev), cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(base + off_tasks, tasks.data(), sizeof(DTask) * (size_t)nen, cudaMemcpyHostToDevice, st));
  NA_CUDA(cudaMemcpyAsync(base + off_order, order.data(), sizeof(int32_t) * (size_t)nen, cudaMemcpyHostToDevice, st));

  int sms = 0;
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = variant_smem(default_variant((int)nm), (int)nm);
  int64_t grid = (int64_t)sms * solver_blocks_per_sm(smem);
  grid = std::min<int64_t>(grid, nen);
  grid = std::min<int64_t>(grid, (int64_t)((kScratchBytes - off_slots) / slot_bytes));
  KParams p;
  std::memset(&p, 0, sizeof(p));
  set_default_variants(p);
  p.o.eta_dev = opts->eta_dev;
  p.o.eta_lead = opts->eta_lead;
  p.o.boltz = opts->boltz;
  p.o.sancho_tol = opts->sancho_tol;
  p.o.sancho_nmax = opts->sancho_nmax;
  p.o.consistent = opts->consistent;
  p.o.want_T = opts->want_T;
  p.devs = (const DDev*)(base + off_dev);
  p.tasks = (const DTask*)(base + off_tasks);
  p.n_tasks = nen;
  p.order = (const int32_t*)(base + off_order);
  p.queue = (int32_t*)base;
  p.work = (double2*)(base + off_slots);
  p.slot_elems = slot_elems_for(nm, nx);
  p.info = (DInfo*)(base + off_info);
  NA_CUDA(launch_solver(p, (int)grid, smem, st));
  std::vector<DInfo> hinfo((size_t)nen);
  NA_CUDA(cudaMemcpyAsync(hinfo.data(), base + off_info, sizeof(DInfo) * (size_t)nen, cudaMemcpyDeviceToHost, st));
  NA_CUDA(cudaStreamSynchronize(st));
#undef NA_CUDA
  int worst = 0;
  for (const DInfo& i : hinfo) worst |= i.status;
  if (info) std::memcpy(info, hinfo.data(), sizeof(DInfo) * (size_t)nen);
  if (worst & RGF_ST_BAD_TASK) return err(RGF_E_ARG, "a task was rejected on the device");
  return worst ? RGF_E_STATUS : RGF_OK;
}
