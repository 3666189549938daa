// Allocation-free variant of the greedy minimum-distance filter.
//
// Some callers cannot allocate device memory while they run. Examples: a host
// that hands this library pointers into a pool it manages and forbids any other
// cudaMalloc, or code running where a device allocation could block or fail
// mid-job (a fixed memory budget agreed up front). tm_find_candidate_indices asks
// such callers for a workspace when more than 2048 points do not fit in shared
// memory. This entry point uses a fixed scratch array compiled into the library
// instead. The array is a file-scope __device__ array, so every GPU that loads
// the library holds it (1.5 MiB) until the process exits.
#include "common.cuh"
#include "peaks.cuh"

#include <cuda.h>  // CUcontext and CUresult types only; the driver calls go through
                   // cudaGetDriverEntryPointByVersion

#include <mutex>
#include <unordered_map>

namespace {

// kept-point coordinates (x, y, z) of the greedy filter, for up to
// TM_NOALLOC_MAX_POINTS points
__device__ __align__(256) int64_t g_candidate_scratch[3 * TM_NOALLOC_MAX_POINTS];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_scratch_mutex;
// CUDA context ID -> device address of g_candidate_scratch in that context. Context
// IDs are unique for the life of the process, so a context created after
// cudaDeviceReset (which unloads this module and loads it again) gets a new entry.
std::unordered_map<unsigned long long, void*> g_scratch_address;

template <typename F>
F driver_function(const char* name) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  if (cudaGetDriverEntryPointByVersion(name, &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(fn);
}

// ID of the calling thread's current context (the device's primary context once the
// runtime has initialised it).
int current_context_id(unsigned long long* id) {
  static const CtxGetCurrentFn get_current = driver_function<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn get_id = driver_function<CtxGetIdFn>("cuCtxGetId");
  TM_REQUIRE(get_current && get_id,
             "tm_find_candidate_indices_noalloc: the driver has no cuCtxGetCurrent/cuCtxGetId");
  CUcontext ctx = nullptr;
  if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, id) != CUDA_SUCCESS) {
    tmb::set_error("tm_find_candidate_indices_noalloc: no current CUDA context");
    return TM_E_CUDA;
  }
  return TM_OK;
}

// Host code cannot pass g_candidate_scratch itself to a kernel: on the host that
// name is a stand-in object, not a device address. Look the address up once per
// device (per context), with that device current.
int scratch_address(void** out) {
  // cudaSetDevice initialises the current device's primary context and makes it current
  // (CUDA 12), without allocating anything
  int dev = 0;
  TM_TRY(tmb::cuda_status(cudaGetDevice(&dev), "tm_find_candidate_indices_noalloc: device"));
  TM_TRY(tmb::cuda_status(cudaSetDevice(dev), "tm_find_candidate_indices_noalloc: device"));
  unsigned long long ctx = 0;
  TM_TRY(current_context_id(&ctx));
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  auto it = g_scratch_address.find(ctx);
  if (it != g_scratch_address.end()) {
    *out = it->second;
    return TM_OK;
  }
  void* ptr = nullptr;
  TM_TRY(tmb::cuda_status(cudaGetSymbolAddress(&ptr, g_candidate_scratch),
                          "tm_find_candidate_indices_noalloc: cudaGetSymbolAddress"));
  g_scratch_address[ctx] = ptr;
  *out = ptr;
  return TM_OK;
}

}  // namespace

extern "C" int tm_find_candidate_indices_noalloc(const int64_t* coords, int n,
                                                 int64_t min_distance, int32_t* out_idx,
                                                 int32_t* out_count, void* stream) {
  TM_REQUIRE(n >= 0, "tm_find_candidate_indices_noalloc: negative point count");
  TM_REQUIRE(n <= TM_NOALLOC_MAX_POINTS,
             "tm_find_candidate_indices_noalloc: %d points exceed the fixed scratch of %d "
             "points; use tm_find_candidate_indices with a workspace",
             n, TM_NOALLOC_MAX_POINTS);
  void* scratch = nullptr;
  TM_TRY(scratch_address(&scratch));
  // The kernel writes each kept point before it reads it back and writes the count
  // itself, so nothing left in the scratch by an earlier call needs clearing.
  return tmb::greedy_nms(coords, n, min_distance, out_idx, out_count, scratch,
                         static_cast<cudaStream_t>(stream));
}
