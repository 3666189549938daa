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

#include <mutex>
#include <unordered_map>

namespace {

// kept-point coordinates (x, y, z) of the greedy filter, for up to
// TM_NOALLOC_MAX_POINTS points
__device__ __align__(256) int64_t g_candidate_scratch[3 * TM_NOALLOC_MAX_POINTS];

std::mutex g_scratch_mutex;
std::unordered_map<int, void*> g_scratch_address;  // device ordinal -> device address

// Host code cannot pass g_candidate_scratch itself to a kernel: on the host that
// name is a stand-in object, not a device address. Look the address up once per
// device, with that device current.
int scratch_address(void** out) {
  int dev = 0;
  TM_TRY(tmb::cuda_status(cudaGetDevice(&dev), "tm_find_candidate_indices_noalloc: device"));
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  auto it = g_scratch_address.find(dev);
  if (it != g_scratch_address.end()) {
    *out = it->second;
    return TM_OK;
  }
  void* ptr = nullptr;
  TM_TRY(tmb::cuda_status(cudaGetSymbolAddress(&ptr, g_candidate_scratch),
                          "tm_find_candidate_indices_noalloc: cudaGetSymbolAddress"));
  g_scratch_address[dev] = ptr;
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
