// dqb_mesolve_dense_noalloc: the dense batched solve for callers that cannot allocate
// device memory.
//
// Some callers have no way to give the library a workspace: code running inside a
// process whose framework has already reserved nearly all of the GPU's memory for its own
// allocator (JAX, for one, preallocates 75% of device memory by default), where a
// cudaMalloc from library code fails or carves memory out of a pool the framework does
// not know about; and deployments whose device-memory footprint is fixed and audited when
// the library is loaded and must not grow afterwards.  For them this entry point takes
// its scratch from a file-scope static device array of DQB_NOALLOC_SCRATCH_BYTES (8 MiB),
// which every GPU that loads the library holds until the process exits, and never calls
// cudaMalloc, cudaFree or an allocating library routine.
//
// The array holds a 256-byte work counter followed by per-CTA slots of
// 9 * NP * NP complex64 (NP = n rounded up to 16, 32 or 64): at n = 64 a slot is
// 288 KiB, so at most 28 instances are in flight at once, fewer than the 148 the
// workspace entry point runs on a B200 -- the results are identical, the throughput lower.
//
// Set-up: the first call on each device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that first call
// before any stream capture.  With lazy module loading (CUDA's default since 12.2) that
// lookup is also when the driver loads this file's module and reserves the array, so the
// first call should precede a framework's preallocation (or set
// CUDA_MODULE_LOADING=EAGER to reserve it at load).  The cache assumes the context of a
// device is never reset; after cudaDeviceReset the cached address would be stale.  Every call shares the one array, and a call leaves its
// contents behind: the work counter is cleared (cudaMemsetAsync on the caller's stream)
// at the start of every call, and the slots need no clearing because every value in them
// is written before it is read.  Calls whose work overlaps on the GPU -- on different
// streams, or from different host threads -- race on the array; serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "dqb_common.cuh"

namespace dqb {
size_t small_slot_bytes(int n);
int small_resident_grid(int n, int K, long long batch);
int small_check_args(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out);
int small_launch_with_scratch(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                              unsigned int* counter, void* slots, int grid, cudaStream_t s);
}  // namespace dqb

namespace {

constexpr size_t kCounterBytes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[DQB_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once per device).
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return DQB_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return DQB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return DQB_ERR_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return DQB_OK;
}

}  // namespace

extern "C" int dqb_mesolve_dense_noalloc(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                         const dqb_outputs* outputs, void* stream) {
  int rc = dqb::small_check_args(problem, options, outputs);
  if (rc) return rc;
  if (problem->batch == 0) return DQB_OK;
  const size_t slot = dqb::small_slot_bytes(problem->n);
  if (slot == 0) return DQB_ERR_UNSUPPORTED;
  if (kCounterBytes + slot > (size_t)DQB_NOALLOC_SCRATCH_BYTES) return DQB_ERR_SCRATCH_TOO_SMALL;
  const long long fit = (long long)(((size_t)DQB_NOALLOC_SCRATCH_BYTES - kCounterBytes) / slot);
  long long grid = dqb::small_resident_grid(problem->n, problem->n_jumps, problem->batch);
  if (grid <= 0) return DQB_ERR_UNSUPPORTED;
  if (grid > fit) grid = fit;
  void* base = nullptr;
  rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(base, 0, kCounterBytes, s) != cudaSuccess) return DQB_ERR_CUDA;
  return dqb::small_launch_with_scratch(problem, options, outputs, (unsigned int*)base,
                                        (char*)base + kCounterBytes, (int)grid, s);
}
